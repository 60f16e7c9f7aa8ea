// One-pass step from the reference layout: LBMNode.update in a single launch.
//
// The reference's update (src/maddening/nodes/lbm.py:899-986) reads f in its
// own layout (*grid, Q), collides every cell, streams, applies the wall swap
// and the faces and returns f_bc with the moments.  Done as two passes
// (k_prepare: f -> p = C(f) into the state planes; k_step: pull p -> f_bc) it
// moves 76 + 76 + 76 + 96 = 324 B per cell.  This kernel moves f once:
//
//   * A block owns a column of the lattice: a tile of TY x TZ cells across
//     the two inner axes, swept along the outer axis plane by plane (D3Q19:
//     tiles over (a1, a2), sweep along a0; D2Q9: row segments of TZ cells
//     along a2, sweep along a1).
//   * Each plane of the column, with a one-cell halo on every side, is moved
//     from the reference layout into a ring of shared-memory slots by the copy
//     engine (1-D bulk asynchronous copies, cp.async.bulk, completion on an
//     mbarrier).  A tile row is copied as whole groups of four cells (a
//     16-byte multiple for Q x 4 B), kTileHalo = 4 cells on each side, with the
//     periodic wrap as separate copies.
//   * Warps have one role each and meet only at mbarriers, never at a block
//     barrier: a producer warp issues the copies of plane P once the slot's
//     previous plane is consumed; collide warps collide plane P in place
//     (every tile and halo cell, k_prepare's arithmetic) once it has landed;
//     output warps, one per 32-cell tile row, pull the collided populations of
//     plane P from slots P - 1, P, P + 1 once P + 1 is collided, apply the
//     wall swap and the faces, take the moments and write f_bc (kOutAoS:
//     staged per warp in shared memory, two staging rows used in turn, and
//     written by a bulk asynchronous store) or collide again and write the
//     next state planes (kOutState: the first step of a rollout).  Collide warps run up
//     to a few planes ahead of the output warps.
//   * A persistent grid walks work items (column, chunk of planes along the
//     sweep); blocks take items with a grid stride in chunk-major order, so
//     neighbouring columns are swept at the same time and the halo rows they
//     share are served by L2.  Each item costs two extra (halo) planes.
//
// Bytes per cell from HBM: 76 (f) + 76 (f_bc) + 20 (moments) + 1 (wall) for
// D3Q19 FP32; the halo re-reads hit L2.  The arithmetic is the two-pass
// path's operation for operation, so the outputs are bit-identical to it.
//
// Requirements (checked on the host): 32-bit IO (FP32, FP16 or BF16
// storage), an a2 extent that is a multiple of 4, f_in (and f_out for
// kOutAoS) 16-byte aligned and not overlapping, no halo-padded block, no
// pipe force.  Every wait is bounded in time and also ends when another warp
// has given up; then the block sets bit 0 of *status, waits (bounded) for its
// own copies in flight and returns.
#pragma once

#include "lbm_kernels.cuh"
#include "lbm_staged.cuh"

namespace lbm {

// Tile shape, warp roles and sweep mapping per lattice.
template <int Q>
struct Sweep;
template <>
struct Sweep<19> {
  static constexpr int TY = 10, TZ = 32;  // tile rows (a1) x row cells (a2)
  static constexpr int HR = 1;            // halo rows
  static constexpr int NCW = 8;           // collide warps, two cells per lane over the
  static constexpr int CPL = 2;           //   (10 + 2) x 40 buffered cells <= 8 x 32 x 2
  static constexpr int MINB = 1;          // resident blocks per SM
  // plane slots: 3 read by the output warps, one being collided, one landing
  // (the ring and two staging rows per output warp fill 226 KB of shared memory)
  static constexpr int SLOTS = 5;
  __host__ __device__ static constexpr int cs(int q) { return Lat<19>::c0(q); }  // sweep
  __host__ __device__ static constexpr int cr(int q) { return Lat<19>::c1(q); }  // rows
};
template <>
struct Sweep<9> {
  static constexpr int TY = 1, TZ = 128;
  static constexpr int HR = 0;
  static constexpr int NCW = 3;  // 136 buffered cells <= 3 x 32 x 2
  static constexpr int CPL = 2;
  static constexpr int MINB = 2;
  static constexpr int SLOTS = 6;  // two planes landing ahead of the collide
  __host__ __device__ static constexpr int cs(int q) { return Lat<9>::c1(q); }
  __host__ __device__ static constexpr int cr(int) { return 0; }
};

constexpr int kTileHalo = 4;   // cells copied on each side of a tile row
constexpr int kMaxTileSlots = 6;  // plane slots of the deepest ring (Sweep<Q>::SLOTS)

template <int Q>
struct TileShape {
  static constexpr int TY = Sweep<Q>::TY, TZ = Sweep<Q>::TZ, HR = Sweep<Q>::HR;
  static constexpr int W = TZ + 2 * kTileHalo;        // cells per buffered row
  static constexpr int RP = TY + 2 * HR;              // buffered rows per plane
  static constexpr int CW = TZ + 2;                   // collided cells per row
  static constexpr int PLANE = RP * W * Q;            // IO elements per plane slot
  static constexpr int NCW = Sweep<Q>::NCW;           // collide warps
  static constexpr int CPL = Sweep<Q>::CPL;           // cells per collide lane
  static constexpr int NOW = TY * TZ / 32;            // output warps (32 cells each)
  static constexpr int NT = 32 * (1 + NCW + NOW);     // + the producer warp
  static_assert(TZ % 32 == 0, "an output warp covers 32 cells of one tile row");
  static_assert(RP <= 32, "one producer lane per buffered row");
  // collide lanes walk every buffered cell (row pitch W), so the 32 cells of
  // a warp access are consecutive in shared memory: no bank conflicts
  static_assert(32 * NCW * CPL >= RP * W, "CPL buffered cells per collide lane and plane");
};

// Barriers and flags of a block, after the slots and the staging rows.
struct TileSync {
  uint64_t full[kMaxTileSlots];      // plane landed (producer arrive + copy bytes)
  uint64_t collided[kMaxTileSlots];  // plane collided (one arrive per collide warp)
  uint64_t consumed[kMaxTileSlots];  // plane read for the last time (one per output warp)
  int abort;                      // a wait gave up
  uint32_t issued;                // planes copied by the producer
  uint32_t landed;                // planes a collide warp has seen land
};

template <int Q, int MODE>
__host__ __device__ constexpr size_t tiled_stage_bytes() {
  return MODE == kOutAoS ? static_cast<size_t>(TileShape<Q>::NOW) * 2 * 32 * Q * 4 : 0;
}
template <int Q, int MODE>
__host__ __device__ constexpr size_t tiled_smem_bytes() {
  return static_cast<size_t>(Sweep<Q>::SLOTS) * TileShape<Q>::PLANE * 4 + tiled_stage_bytes<Q, MODE>() +
         sizeof(TileSync);
}

// Host-computed geometry of the sweep.
struct TileGeo {
  uint32_t NS, NR;        // planes along the sweep axis; rows per plane
  uint32_t SS, SR;        // cell strides of the sweep and row axes
  uint32_t ncolz, ncol;   // tiles along a2; tiles per plane
  uint32_t chunk, items;  // planes per work item; work items = ncol x chunks
  uint64_t wait_ns;       // a wait gives up after this long (global timer)
  uint32_t no_copy;       // test hook: barriers armed, no copies issued
};

// One plane of a work item: j = 0 and j = nv + 1 are the halo planes.  The
// item's position is cached when the item starts.
struct PlaneRef {
  uint32_t item, j, nv;
  uint32_t k0;        // first plane of the chunk (sweep coordinate of j = 1)
  uint32_t y0, z0;    // first tile row / cell
  uint32_t tyv, tzv;  // tile rows / cells inside the lattice
};

template <int Q>
__device__ __forceinline__ void plane_first(const StepArgs& a, const TileGeo& t, uint32_t item,
                                            PlaneRef& p) {
  using T = TileShape<Q>;
  p.item = item;
  p.j = 0;
  if (item >= t.items) return;
  const uint32_t col = item % t.ncol;
  p.k0 = (item / t.ncol) * t.chunk;
  p.nv = t.NS - p.k0 < t.chunk ? t.NS - p.k0 : t.chunk;
  p.y0 = (col / t.ncolz) * T::TY;
  p.z0 = (col % t.ncolz) * T::TZ;
  p.tyv = t.NR - p.y0 < static_cast<uint32_t>(T::TY) ? t.NR - p.y0 : T::TY;
  p.tzv = a.g.n2 - p.z0 < static_cast<uint32_t>(T::TZ) ? a.g.n2 - p.z0 : T::TZ;
}
template <int Q>
__device__ __forceinline__ void plane_next(const StepArgs& a, const TileGeo& t, PlaneRef& p) {
  if (p.item >= t.items) return;
  if (++p.j == p.nv + 2) plane_first<Q>(a, t, p.item + gridDim.x, p);
}
// Sweep coordinate of the plane (periodic wrap for the halo planes).
__device__ __forceinline__ uint32_t plane_s(const TileGeo& t, const PlaneRef& p) {
  return wrapu(static_cast<int>(p.k0 + p.j) - 1, t.NS);
}

// Producer warp: lane 0 arms `bar` with the bytes of one plane (tile rows with
// their halo), then lane rr copies buffered row rr into buf, so the copies of a
// plane are issued together rather than one after another.
template <int Q>
__device__ __forceinline__ void tiled_issue(const StepArgs& a, const TileGeo& t,
                                            const PlaneRef& p, float* buf, uint64_t* bar,
                                            uint32_t lane) {
  using T = TileShape<Q>;
  const uint32_t ps = plane_s(t, p);
  const uint32_t nrow = p.tyv + 2 * T::HR;
  constexpr uint32_t cellb = Q * 4;
  if (lane == 0) mbar_arrive_expect_tx(bar, nrow * (p.tzv + 2 * kTileHalo) * cellb);
  __syncwarp();
  const uint32_t rr = lane;
  if (t.no_copy || rr >= nrow) return;
  const float* f = static_cast<const float*>(a.f_in);
  const uint32_t n2 = a.g.n2;
  const uint32_t r = wrapu(static_cast<int>(p.y0 + rr) - T::HR, t.NR);
  const size_t rowc = static_cast<size_t>(ps) * t.SS + static_cast<size_t>(r) * t.SR;
  float* dst = buf + static_cast<size_t>(rr) * T::W * Q;
  uint32_t col = 0;  // buffer cell of the next copy
  uint32_t z = p.z0 - kTileHalo;
  if (p.z0 == 0) {  // left halo group wraps to the end of the row
    bulk_copy_g2s(dst, f + (rowc + n2 - kTileHalo) * Q, kTileHalo * cellb, bar);
    col = kTileHalo;
    z = 0;
  }
  const bool wrap_r = p.z0 + p.tzv == n2;
  const uint32_t zend = wrap_r ? n2 : p.z0 + p.tzv + kTileHalo;
  bulk_copy_g2s(dst + static_cast<size_t>(col) * Q, f + (rowc + z) * Q, (zend - z) * cellb,
                bar);
  if (wrap_r)  // right halo group wraps to the start of the row
    bulk_copy_g2s(dst + static_cast<size_t>(kTileHalo + p.tzv) * Q, f + rowc * Q,
                  kTileHalo * cellb, bar);
}

// p = C(f) of the reference state of cell c (k_prepare's arithmetic), with the
// 16-bit storage rounding applied and undone: d holds the values the state
// planes would return.
template <int Q, class S, bool FORCE>
__device__ __forceinline__ void collide_ref(const StepArgs& a, uint32_t c, float (&d)[Q]) {
  using R = float;
  R F[3] = {0, 0, 0};
  if (FORCE) {
    if (a.force_mode == 2) load_force<Q, float>(a.force_field, c, F);
    else uniform_force<Q, R>(a, F);
  }
  const Mom<R> m = moments<Q, R, FORCE>(d, F, true);
  collide<Q, R, FORCE>(d, m, F, static_cast<R>(a.omega), static_cast<R>(a.guo_c));
  if constexpr (sizeof(S) == 2) {
    const uint32_t seed = sr_seed(c, m.u[0], m.u[1], m.u[2], m.rd);
#pragma unroll
    for (int q = 0; q < Q; ++q) d[q] = to_r(sr_one<S>(d[q], sr_bits(seed, d[q])));
  }
}

// Population qs of p = C(f) at cell c, from the reference state in global
// memory (zero-gradient faces reach cells outside the buffered planes).
template <int Q, class S, bool FORCE>
__device__ __noinline__ float collided_pop(const StepArgs& a, uint32_t c, int qs) {
  const float* fi = static_cast<const float*>(a.f_in) + static_cast<size_t>(c) * Q;
  float d[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) d[q] = to_offset<Q, float>(__ldg(fi + q), q);
  collide_ref<Q, S, FORCE>(a, c, d);
  float v = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q)
    if (q == qs) v = d[q];
  return v;
}

// Zero-gradient face of the one-pass step: unknown q <- f_bc of the cell one
// inwards, its pulled (or wall-swapped) population recomputed from f_in.
template <int Q, class S, bool FORCE>
__device__ __forceinline__ void face_zero_gradient_ref(float (&d)[Q], const StepArgs& a, int fi,
                                                       const Cell& x) {
  const Geo& g = a.g;
  const FaceK& fc = a.face[fi];
  const int ax = fc.axis;
  const int st = fc.side == 0 ? 1 : -1;
  const int n0 = static_cast<int>(x.i0) + (ax == 0 ? st : 0);
  const int n1 = static_cast<int>(x.i1) + (ax == 1 ? st : 0);
  const int n2 = static_cast<int>(x.k) + (ax == 2 ? st : 0);
  const bool wl =
      a.wall != nullptr && a.wall[(static_cast<uint32_t>(n0) * g.n1 + n1) * g.n2 + n2] != 0;
  const int s = wl ? 1 : -1;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = fc.side == 0 ? (cq > 0) : (cq < 0);
    if (!unknown) continue;
    const uint32_t j0 = wrapu(n0 + s * Lat<Q>::c0(q), g.n0);
    const uint32_t j1 = wrapu(n1 + s * Lat<Q>::c1(q), g.n1);
    const uint32_t j2 = wrapu(n2 + s * Lat<Q>::c2(q), g.n2);
    d[q] = collided_pop<Q, S, FORCE>(a, (j0 * g.n1 + j1) * g.n2 + j2, wl ? Lat<Q>::opp(q) : q);
  }
}

// Wall swap and faces of a pulled cell (apply_bc with the zero-gradient
// neighbour taken from the reference state).  The swap is a select on every
// pair and the faces are entered only when a cell of the warp lies on one:
// fewer branches in the output warps' path than apply_bc's.
template <int Q, class S, bool FACES, bool FORCE>
__device__ __forceinline__ void apply_bc_ref(const StepArgs& a, const Cell& x, bool wall,
                                             float (&d)[Q]) {
#pragma unroll
  for (int q = 1; q < Q; ++q) {
    if (q < Lat<Q>::opp(q)) {
      const float u = d[q], v = d[Lat<Q>::opp(q)];
      d[q] = wall ? v : u;
      d[Lat<Q>::opp(q)] = wall ? u : v;
    }
  }
  if constexpr (FACES) {
    const Geo& g = a.g;
    uint32_t on = 0;
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
      const FaceK& fc = a.face[fi];
      const uint32_t coord = fc.axis == 0 ? x.i0 : (fc.axis == 1 ? x.i1 : x.k);
      const uint32_t nax = fc.axis == 0 ? g.n0 : (fc.axis == 1 ? g.n1 : g.n2);
      if (fc.kind != kFaceNone && coord == (fc.side == 0 ? 0u : nax - 1)) on |= 1u << fi;
    }
    if (wall) on = 0;
    if (__any_sync(__activemask(), on != 0)) {
#pragma unroll
      for (int fi = 0; fi < 2; ++fi) {
        if (!((on >> fi) & 1u)) continue;
        const FaceK& fc = a.face[fi];
        if (fc.kind == kFacePressure) face_pressure<Q, float>(d, a, fi);
        else if (fc.kind == kFaceVelocity) face_velocity<Q, float>(d, a, fi);
        else face_zero_gradient_ref<Q, S, FORCE>(d, a, fi, x);
      }
    }
  }
}

// A wall byte, loaded where the source places it: the output warps fetch the
// next plane's byte one plane ahead, and a volatile load is neither moved
// towards its use nor repeated there by the compiler.
__device__ __forceinline__ uint8_t ld_wall(const uint8_t* p) {
  uint16_t v;
  asm volatile("ld.global.nc.u8 %0, [%1];" : "=h"(v) : "l"(p));
  return static_cast<uint8_t>(v);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// try_wait that suspends the thread until the phase completes or about 20 us
// pass (a hint: the hardware may return earlier), so a waiting warp takes few
// issue slots from the working ones.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
      : "memory");
  return ok != 0;
}

// Wait bounded by wall time (limit_ns of the global timer) that also ends when
// another warp of the block has given up (*abort set); a wait that runs out
// sets *abort itself.  Between polls the warp sleeps, up to max_sleep_ns, so
// that waiting warps leave the issue slots to the working ones.
__device__ __forceinline__ bool tile_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns,
                                          volatile int* abort, uint32_t max_sleep_ns) {
  if (mbar_try_wait_sleep(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  uint32_t sleep = 32;
  for (;;) {
    if (mbar_try_wait_sleep(bar, parity)) return true;
    if (*abort) return false;
    if (globaltimer_ns() - t0 > limit_ns) break;
    __nanosleep(sleep);
    sleep = sleep < max_sleep_ns ? 2 * sleep : max_sleep_ns;
  }
  *abort = 1;
  return false;
}

template <int Q, class S, int MODE, bool FACES, bool FORCE>
__global__ void __launch_bounds__(TileShape<Q>::NT, Sweep<Q>::MINB)
    k_tiled(const __grid_constant__ StepArgs a, const __grid_constant__ TileGeo t) {
  using T = TileShape<Q>;
  using R = float;
  static_assert(MODE == kOutAoS || MODE == kOutState, "f_bc out or the next state out");
  constexpr uint32_t S_ = Sweep<Q>::SLOTS;
  static_assert(Sweep<Q>::SLOTS >= 5 && Sweep<Q>::SLOTS <= kMaxTileSlots, "ring depth");
  extern __shared__ __align__(128) unsigned char smem[];
  float* planes = reinterpret_cast<float*>(smem);
  float* stage = planes + static_cast<size_t>(S_) * T::PLANE;
  TileSync* sync = reinterpret_cast<TileSync*>(
      smem + static_cast<size_t>(S_) * T::PLANE * 4 + tiled_stage_bytes<Q, MODE>());
  volatile int* abort = &sync->abort;
  const Geo& g = a.g;
  const uint32_t tid = threadIdx.x;
  const uint32_t lane = tid & 31u, warp = tid >> 5;

  if (tid == 0) {
    for (uint32_t s = 0; s < S_; ++s) {
      mbar_init(&sync->full[s], 1);
      mbar_init(&sync->collided[s], T::NCW);
      mbar_init(&sync->consumed[s], T::NOW);
    }
    sync->abort = 0;
    sync->issued = 0;
    sync->landed = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == 0) {
    // ---- producer: copy plane P into slot P % S once plane P - S is consumed
    {
      PlaneRef L;
      plane_first<Q>(a, t, blockIdx.x, L);
      uint32_t P = 0;
      for (; L.item < t.items; plane_next<Q>(a, t, L), ++P) {
        const uint32_t sl = P % S_;
        const bool ok = P < S_ ||
                        tile_wait(&sync->consumed[sl], (P / S_ - 1) & 1u, t.wait_ns, abort, 1024);
        if (!__all_sync(0xffffffffu, ok)) break;
        fence_proxy_async_smem();
        tiled_issue<Q>(a, t, L, planes + static_cast<size_t>(sl) * T::PLANE, &sync->full[sl],
                       lane);
      }
      if (lane == 0) sync->issued = P;
    }
  } else if (warp <= static_cast<uint32_t>(T::NCW)) {
    // ---- collide warps: plane P in place once it has landed; lane cells
    // m_k = lane + 32 (warp - 1 + k NCW), k < CPL, of the buffered cells (row
    // pitch W; the collided ones are columns kTileHalo - 1 .. kTileHalo + TZ),
    // their loads issued together
    using T2 = TileShape<Q>;
    uint32_t soff[T2::CPL], rr[T2::CPL], cc[T2::CPL], rz[T2::CPL];
    bool mine[T2::CPL];
#pragma unroll
    for (int k = 0; k < T2::CPL; ++k) {
      const uint32_t m = (warp - 1 + k * T2::NCW) * 32 + lane;
      rr[k] = m / T::W;
      cc[k] = m % T::W - (kTileHalo - 1);  // wraps above CW for the unused columns
      soff[k] = m * Q;                      // its place in a slot
      mine[k] = false;
      rz[k] = 0;
    }
    PlaneRef C;
    plane_first<Q>(a, t, blockIdx.x, C);
    uint32_t P = 0, item = ~0u;
    for (; C.item < t.items; plane_next<Q>(a, t, C), ++P) {
      if (C.item != item) {  // a new work item: the lane cells' rows and columns
        item = C.item;
#pragma unroll
        for (int k = 0; k < T2::CPL; ++k) {
          mine[k] = rr[k] < C.tyv + 2 * T::HR && cc[k] < C.tzv + 2;
          rz[k] = wrapu(static_cast<int>(C.y0 + rr[k]) - T::HR, t.NR) * t.SR +
                  wrapu(static_cast<int>(C.z0 + cc[k]) - 1, g.n2);
        }
      }
      const uint32_t sl = P % S_;
      const bool ok = tile_wait(&sync->full[sl], (P / S_) & 1u, t.wait_ns, abort, 1024);
      if (!__all_sync(0xffffffffu, ok)) break;
      if (lane == 0) atomicMax(&sync->landed, P + 1);
      float* slot = planes + static_cast<size_t>(sl) * T::PLANE;
      const uint32_t cs0 = plane_s(t, C) * t.SS;
      R d[T2::CPL][Q];
#pragma unroll
      for (int k = 0; k < T2::CPL; ++k) {
        if (mine[k]) {
#pragma unroll
          for (int q = 0; q < Q; ++q) d[k][q] = to_offset<Q, R>(slot[soff[k] + q], q);
        }
      }
#pragma unroll
      for (int k = 0; k < T2::CPL; ++k) {
        if (mine[k]) {
          collide_ref<Q, S, FORCE>(a, cs0 + rz[k], d[k]);
#pragma unroll
          for (int q = 0; q < Q; ++q) slot[soff[k] + q] = d[k][q];
        }
      }
      fence_proxy_async_smem();  // before the slot is refilled by a copy
      __syncwarp();
      if (lane == 0) mbar_arrive(&sync->collided[sl]);
    }
  } else {
    // ---- output warps: tile row `ty` of plane P once P + 1 is collided
    const uint32_t ow = warp - 1 - T::NCW;
    const uint32_t ty = ow / (T::TZ / 32), tz = (ow % (T::TZ / 32)) * 32 + lane;
    // this warp's two staging rows, used in turn: a plane's store may still be
    // reading one while the next plane is staged in the other
    float* const wst2 = stage + static_cast<size_t>(ow) * 2 * 32 * Q;
    uint32_t nstore = 0;  // bulk stores this warp has issued
    const uint32_t off = ((ty + T::HR) * T::W + kTileHalo + tz) * Q;  // own cell in a slot
    PlaneRef O;
    plane_first<Q>(a, t, blockIdx.x, O);
    uint32_t P = 0;
    uint32_t wnext_c = ~0u;  // cell whose wall byte was fetched one plane ahead
    uint8_t wnext = 0;
    for (; O.item < t.items; plane_next<Q>(a, t, O), ++P) {
      if (O.j < 1 || O.j > O.nv) continue;
      const uint32_t sn = (P + 1) % S_;
      const bool ok =
          tile_wait(&sync->collided[sn], ((P + 1) / S_) & 1u, t.wait_ns, abort, 64);
      if (!__all_sync(0xffffffffu, ok)) break;
      const uint32_t ps = plane_s(t, O);
      const bool act = ty < O.tyv && tz < O.tzv;
      Cell x;
      if (Lat<Q>::D == 3) {
        x.i0 = ps;
        x.i1 = O.y0 + ty;
      } else {
        x.i0 = 0;
        x.i1 = ps;
      }
      x.k = O.z0 + tz;
      x.c = ps * t.SS + (O.y0 + ty) * t.SR + x.k;
      x.row = x.c - x.k;
      x.srow = x.row;
      float* const wst = wst2 + (nstore & 1u) * 32 * Q;
      if constexpr (MODE == kOutAoS) {
        // the store before the last one has finished reading this staging row
        if (lane == 0) bulk_wait_read_1();
        __syncwarp();
      }
      uint8_t wb = 0;
      if (act && a.wall != nullptr) {
        wb = x.c == wnext_c ? wnext : ld_wall(a.wall + x.c);
        if (O.j < O.nv) {  // the same lane's cell of the next plane of this item
          wnext_c = x.c + t.SS;
          wnext = ld_wall(a.wall + wnext_c);
        }
      }
      R d[Q];
      R F[3] = {0, 0, 0};
      Mom<R> mo;
      const bool wall = wb != 0;
      if (act) {
        // the three planes of the pull: x - e_q lies in plane P - c_s(q)
        const float* pm = planes + static_cast<size_t>((P + S_ - 1) % S_) * T::PLANE + off;
        const float* p0 = planes + static_cast<size_t>(P % S_) * T::PLANE + off;
        const float* pp = planes + static_cast<size_t>(sn) * T::PLANE + off;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const int cs = Sweep<Q>::cs(q);
          const float* base = cs > 0 ? pm : (cs < 0 ? pp : p0);
          d[q] = base[(-Sweep<Q>::cr(q) * T::W - Lat<Q>::c2(q)) * Q + q];
        }
        if (FORCE) {
          if (a.force_mode == 2) load_force<Q, float>(a.force_field, x.c, F);
          else uniform_force<Q, R>(a, F);
        }
        apply_bc_ref<Q, S, FACES, FORCE>(a, x, wall, d);
        mo = moments<Q, R, FORCE>(d, F, true);
        if constexpr (MODE == kOutAoS) {
          float* row = wst + lane * Q;
#pragma unroll
          for (int q = 0; q < Q; ++q) row[q] = from_offset<Q, R>(d[q], q);
        }
      }
      if constexpr (MODE == kOutAoS) {
        // The warp's cells are a prefix of one contiguous run of the output.
        // The proxy fence comes before this warp's global stores of the
        // moments, so that it waits only for the staging writes.
        const uint32_t nvalid = __popc(__ballot_sync(0xffffffffu, act));
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0 && nvalid > 0)
          bulk_store_s2g(static_cast<float*>(a.f_out) + static_cast<size_t>(x.c) * Q, wst,
                         nvalid * Q * 4);
        nstore += nvalid > 0 ? 1u : 0u;
      }
      if (act) {
        store_moments<Q, float>(a, x.c, mo, wall);
        if constexpr (MODE == kOutState) {
          collide<Q, R, FORCE>(d, mo, F, static_cast<R>(a.omega), static_cast<R>(a.guo_c));
          S* out = static_cast<S*>(a.pout) + x.srow + x.k;
          if constexpr (sizeof(S) == 2) {
            const uint32_t seed = sr_seed(x.c, mo.u[0], mo.u[1], mo.u[2], mo.rd);
#pragma unroll
            for (int q = 0; q < Q; ++q)
              out[static_cast<uint32_t>(q) * g.pstride] = sr_one<S>(d[q], sr_bits(seed, d[q]));
          } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) out[static_cast<uint32_t>(q) * g.pstride] = d[q];
          }
        }
      }
      __syncwarp();
      if (lane == 0) {
        // plane P - 1 has had its last reader; at the end of an item, P and P + 1 too
        mbar_arrive(&sync->consumed[(P + S_ - 1) % S_]);
        if (O.j == O.nv) {
          mbar_arrive(&sync->consumed[P % S_]);
          mbar_arrive(&sync->consumed[sn]);
        }
      }
    }
    if constexpr (MODE == kOutAoS) {
      if (lane == 0) bulk_wait_all();
    }
  }

  __syncthreads();
  if (tid == 0 && sync->abort) {
    atomicOr(a.status, 1);
    // copies issued and not seen landing: wait for them (bounded) before exit
    sync->abort = 0;
    for (uint32_t P = sync->landed; P < sync->issued; ++P)
      if (!tile_wait(&sync->full[P % S_], (P / S_) & 1u, t.wait_ns, abort, 512)) break;
  }
}

}  // namespace lbm
