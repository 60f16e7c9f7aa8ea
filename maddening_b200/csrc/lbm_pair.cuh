// Paired-cell fused step: each thread updates two neighbouring cells (k, k+1)
// of one row, reading and writing every population plane as one 32-bit word
// (two 16-bit offsets) or one 64-bit word (two FP32 offsets).
//
// Why: with 16-bit storage a one-cell-per-thread step keeps only 19 x 2 B of
// loads in flight per thread, too little to cover HBM latency at the
// occupancy its registers allow, and it spends an address computation, a
// conversion and a memory instruction on every 2-byte value.  Pairs double
// the bytes in flight per thread, pack each output pair with one conversion
// and halve the memory instructions.
//
// Block layout: a block of W warps covers 64 W consecutive cells of one row
// (blockIdx.x = row i0 * n1 + i1, blockIdx.y = segment along the row), so the
// row coordinates and the 19 source-row base pointers are block-uniform.  Lane
// l of a warp owns the aligned pair (k, k+1), k = first + 2 l.  The pull
// along the contiguous axis:
//   c2 =  0: both cells read the thread's own pair;
//   c2 = +1: cell k reads k - 1, the high half of the pair before (a second
//            aligned word, wrapped at the row start; the neighbouring lane
//            loads the same line, so it hits L1); cell k+1 reads the low half
//            of its own pair;
//   c2 = -1: mirror image (the pair after, wrapped at the row end).
// After the pull each cell runs exactly the arithmetic of the one-cell step
// (wall swap -> faces -> moments -> collide), so the results are
// bit-identical; the wall swap is skipped by warps without a wall cell and the
// face checks by pairs that cannot touch a face.
//
// A second form (k_step_gpair) takes any even row length: pairs follow the
// instance-wide cell index and each lane finds its own row.
//
// Requirements (checked on the host): an even contiguous extent n2 (a multiple
// of 64 W for the row-segment form), state planes and the wall mask aligned for
// the pair width.  Used for the state-to-state steps of a rollout; the other
// modes keep the one-cell kernels.
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

template <class S>
struct PairT;

template <>
struct PairT<__half> {
  using P = uint32_t;
  static __device__ __forceinline__ P ld(const __half* p) {
    return __ldg(reinterpret_cast<const unsigned int*>(p));
  }
  static __device__ __forceinline__ float lo(P v) {
    return __low2float(*reinterpret_cast<const __half2*>(&v));
  }
  static __device__ __forceinline__ float hi(P v) {
    return __high2float(*reinterpret_cast<const __half2*>(&v));
  }
};

template <>
struct PairT<__nv_bfloat16> {
  using P = uint32_t;
  static __device__ __forceinline__ P ld(const __nv_bfloat16* p) {
    return __ldg(reinterpret_cast<const unsigned int*>(p));
  }
  static __device__ __forceinline__ float lo(P v) { return __uint_as_float(v << 16); }
  static __device__ __forceinline__ float hi(P v) { return __uint_as_float(v & 0xffff0000u); }
};

template <>
struct PairT<float> {
  using P = float2;
  static __device__ __forceinline__ P ld(const float* p) {
    return __ldg(reinterpret_cast<const float2*>(p));
  }
  static __device__ __forceinline__ float lo(P v) { return v.x; }
  static __device__ __forceinline__ float hi(P v) { return v.y; }
  static __device__ __forceinline__ void st(float* p, float a, float b) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
};

// Resident warps per SM the register budgets are set for (a B200 sweep of
// 20-32: the row-segment form is fastest at 32 warps despite a few spilled
// registers, the instance-wide form at 28).
#ifndef LBM_PAIR_MIN_WARPS
#define LBM_PAIR_MIN_WARPS 32
#endif
#ifndef LBM_GPAIR_MIN_WARPS
#define LBM_GPAIR_MIN_WARPS 28
#endif
constexpr int kPairMinWarps = LBM_PAIR_MIN_WARPS;
constexpr int kGPairMinWarps = LBM_GPAIR_MIN_WARPS;

// Moments and collide of one cell whose f_bc populations are in d; `real` =
// false for the padding cell of a padded row (its result is never read).
// Returns the cell's stochastic-rounding seed (16-bit storage; else 0).
template <int Q, class S, bool FORCE>
__device__ __forceinline__ uint32_t pair_cell(const StepArgs& a, const Cell& x, float (&d)[Q],
                                              bool real = true) {
  using IO = typename StoreT<S>::IO;
  float F[3] = {0, 0, 0};
  if (FORCE) {
    if (a.force_mode == 2) {
      if (real) load_force<Q, IO>(a.force_field, x.c, F);
    } else {
      uniform_force<Q, float>(a, F);
    }
  }
  const Mom<float> m = moments<Q, float, FORCE>(d, F);
  collide<Q, float, FORCE>(d, m, F, static_cast<float>(a.omega), static_cast<float>(a.guo_c));
  if constexpr (sizeof(S) == 2) return sr_seed(x.c, m.u[0], m.u[1], m.u[2], m.rd);
  else return 0u;
}

// Everything after the plane loads of one thread's pair (k, k+1) of row
// `rbase` (reference layout; `sbase` in the state planes): v[q] the pair word
// at (k, k+1) of the source row of direction q, e[q] the word of the pair
// before (c2 > 0: cell k pulls k - 1) or after (c2 < 0: cell k + 1 pulls
// k + 2), periodic along the row.  In a padded row (odd n2, state rows of
// n2 + 1) the last pair is (n2 - 1, padding): cell 0 finds n2 - 1 and cell
// n2 - 1 finds 0 in the LOW half of their neighbour word.  All 32 lanes of the
// warp must call it (vote); `store` = false for lanes that only pad the warp.
// PAD: the state rows are padded (compile time: the checks cost instructions).
template <int Q, class S, bool FACES, bool FORCE, bool PAD>
__device__ __forceinline__ void pair_finish(const StepArgs& a, uint32_t i0, uint32_t i1,
                                            uint32_t k, uint32_t rbase, uint32_t sbase,
                                            const typename PairT<S>::P (&v)[Q],
                                            const typename PairT<S>::P (&e)[Q], bool store) {
  using PT = PairT<S>;
  const Geo& g = a.g;
  const bool first = PAD && k == 0;
  const bool last = PAD && k + 1 == g.n2;  // cell b is the padding cell
  float da[Q], db[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c2 = Lat<Q>::c2(q);
    if (c2 == 0) {
      da[q] = PT::lo(v[q]);
      db[q] = PT::hi(v[q]);
    } else if (c2 > 0) {
      da[q] = first ? PT::lo(e[q]) : PT::hi(e[q]);
      db[q] = PT::lo(v[q]);
    } else {
      da[q] = last ? PT::lo(e[q]) : PT::hi(v[q]);
      db[q] = PT::lo(e[q]);
    }
  }
  bool wa = false, wb = false;
  if (a.wall != nullptr) {
    if constexpr (PAD) {  // odd rows: the two wall bytes are not 2-byte aligned
      wa = __ldg(a.wall + rbase + k) != 0;
      wb = !last && __ldg(a.wall + rbase + k + 1) != 0;
    } else {
      const uint32_t w2 = __ldg(reinterpret_cast<const unsigned short*>(a.wall + rbase + k));
      wa = (w2 & 0xffu) != 0;
      wb = (w2 >> 8) != 0;
    }
  }
  Cell xa, xb;
  xa.c = rbase + k;
  xa.i0 = i0;
  xa.i1 = i1;
  xa.k = k;
  xa.row = rbase;
  xa.srow = sbase;
  xb = xa;
  xb.c = xa.c + 1;
  xb.k = k + 1;
  // Wall swap only in warps that hold a wall cell (obstacles are clustered).
  if (__any_sync(0xffffffffu, wa || wb)) {
    if (wa) wall_swap<Q>(da);
    if (wb) wall_swap<Q>(db);
  }
  if constexpr (FACES) {
    // Only pairs on a face plane run the face code: rows on faces of axes 0
    // and 1, the first and the last pair of a row on faces of the contiguous axis.
    bool near = false;
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
      const FaceK& fc = a.face[fi];
      if (fc.kind == kFaceNone) continue;
      const uint32_t ins = a.face_inset;
      if (fc.axis == 0) near |= i0 == (fc.side == 0 ? ins : g.n0 - 1 - ins);
      else if (fc.axis == 1) near |= i1 == (fc.side == 0 ? ins : g.n1 - 1 - ins);
      else near |= (fc.side == 0 ? ins : g.n2 - 1 - ins) - k <= 1u;  // k or k + 1
    }
    if (near) {
      if (!wa) apply_faces<Q, S>(a, xa, da);
      if (!wb && !last) apply_faces<Q, S>(a, xb, db);  // never on the padding cell
    }
  }
  const uint32_t sa = pair_cell<Q, S, FORCE>(a, xa, da);
  const uint32_t sb = pair_cell<Q, S, FORCE>(a, xb, db, !last);
  if (!store) return;
  S* pout = static_cast<S*>(a.pout);
  const uint32_t s2 = sr_pair(sa, sb);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    S* dst = pout + (static_cast<uint32_t>(q) * g.pstride + sbase + k);
    if constexpr (sizeof(S) == 2)
      *reinterpret_cast<uint32_t*>(dst) = sr_two<S>(da[q], db[q], s2);
    else
      PT::st(dst, da[q], db[q]);
  }
}

// Row-segment form: rows of 64 W cells or a multiple (see the header comment).
template <int Q, class S, bool FACES, bool FORCE, int W>
__global__ void __launch_bounds__(32 * W, kPairMinWarps / W)
    k_step_pair(const __grid_constant__ StepArgs a) {
  using PT = PairT<S>;
  using P = typename PT::P;
  const Geo& g = a.g;
  const uint32_t row = blockIdx.x;
  const uint32_t i0 = fdiv(row, g.div_n1);
  const uint32_t i1 = row - i0 * g.n1;
  const uint32_t k = blockIdx.y * (64u * W) + 2u * threadIdx.x;
  // pair before / after this thread's pair (periodic along the row)
  const uint32_t kprev = (k == 0 ? g.n2 : k) - 2u;
  const uint32_t knext = k + 2u == g.n2 ? 0u : k + 2u;
  // source rows of the pull x - e_q (periodic)
  const uint32_t i0m = i0 == 0 ? g.n0 - 1 : i0 - 1, i0p = i0 + 1 == g.n0 ? 0u : i0 + 1;
  const uint32_t i1m = i1 == 0 ? g.n1 - 1 : i1 - 1, i1p = i1 + 1 == g.n1 ? 0u : i1 + 1;

  const S* pin = static_cast<const S*>(a.pin);
  P v[Q];
  P e[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q), c2 = Lat<Q>::c2(q);
    const uint32_t s0 = c0 > 0 ? i0m : (c0 < 0 ? i0p : i0);
    const uint32_t s1 = c1 > 0 ? i1m : (c1 < 0 ? i1p : i1);
    const S* base = pin + (static_cast<uint32_t>(q) * g.pstride + (s0 * g.n1 + s1) * g.rstride);
    v[q] = PT::ld(base + k);
    if (c2 > 0) e[q] = PT::ld(base + kprev);
    if (c2 < 0) e[q] = PT::ld(base + knext);
  }
  pair_finish<Q, S, FACES, FORCE, false>(a, i0, i1, k, row * g.n2, row * g.rstride, v, e, true);
}

// ---------------------------------------------------------------------------
// Four cells per thread (16-bit storage)
// ---------------------------------------------------------------------------
// With 16-bit offsets a pair still leaves each thread with few bytes in
// flight and a large share of per-cell overhead (addresses, memory
// instructions, the wall load, the vote): a D2Q9 cell carries only 9 x 2 B.  Here lane l of a warp owns cells
// k..k+3 (k = first + 4 l) of one row and moves each plane as one 64-bit word
// (four 16-bit offsets); the pull along the row takes the neighbour of cell k
// (c2 = +1) or of cell k+3 (c2 = -1) from the aligned 32-bit word before /
// after the quad.  Every cell then runs the one-cell arithmetic (bit-identical
// results).  Block: W warps = 128 W consecutive cells of one row; rows of a
// multiple of 128 W cells.
template <class S>
struct QuadT {
  static __device__ __forceinline__ uint2 ld(const S* p) {
    return __ldg(reinterpret_cast<const uint2*>(p));
  }
};

// Resident warps the D3Q19 four-cell budget is set for (B200 sweep at 256^3,
// FP16: 16 warps 78.1k, 20 warps 79.4k, 22 / 24 warps 69k MLUPS -- at 20 the 96
// registers spill a few bytes, beyond it the spills cost more than the warps).
#ifndef LBM_QUAD19_MIN_WARPS
#define LBM_QUAD19_MIN_WARPS 20
#endif
// D2Q9 four-cell budget (B200 sweep, 4096^2 channel FP16: 24 / 32 / 40 / 48
// resident warps 134.9k / 138.5k / 125.0k / 98.9k MLUPS).
#ifndef LBM_QUAD9_MIN_WARPS
#define LBM_QUAD9_MIN_WARPS LBM_PAIR_MIN_WARPS
#endif
template <int Q>
constexpr int quad_min_warps() { return Q == 19 ? LBM_QUAD19_MIN_WARPS : LBM_QUAD9_MIN_WARPS; }

// The populations of quad (k..k+3) of source row `base` pulled along the row:
// kprev / knext the aligned 32-bit words holding cells k - 1 / k + 4
// (periodic).
template <int Q, class S>
__device__ __forceinline__ void quad_pull(const S* base, int q, uint32_t k, uint32_t kprev,
                                          uint32_t knext, float (&d)[4][Q]) {
  using PT = PairT<S>;
  const int c2 = Lat<Q>::c2(q);
  const uint2 v = QuadT<S>::ld(base + k);
  if (c2 == 0) {
    d[0][q] = PT::lo(v.x);
    d[1][q] = PT::hi(v.x);
    d[2][q] = PT::lo(v.y);
    d[3][q] = PT::hi(v.y);
  } else if (c2 > 0) {  // cell j pulls j - 1
    d[0][q] = PT::hi(PT::ld(base + kprev));
    d[1][q] = PT::lo(v.x);
    d[2][q] = PT::hi(v.x);
    d[3][q] = PT::lo(v.y);
  } else {  // cell j pulls j + 1
    d[0][q] = PT::hi(v.x);
    d[1][q] = PT::lo(v.y);
    d[2][q] = PT::hi(v.y);
    d[3][q] = PT::lo(PT::ld(base + knext));
  }
}

// Everything after the pull of quad (k..k+3) of row (i0, i1): wall swap,
// faces, moments and collide of each cell, packed stores.  All 32 lanes of the
// warp call it (vote); `store` = false for lanes that only pad the warp.
template <int Q, class S, bool FACES, bool FORCE>
__device__ __forceinline__ void quad_finish(const StepArgs& a, uint32_t i0, uint32_t i1,
                                            uint32_t k, uint32_t row, float (&d)[4][Q],
                                            bool store) {
  const Geo& g = a.g;
  const uint32_t rbase = row * g.n2, sbase = row * g.rstride;
  bool w[4] = {false, false, false, false};
  if (a.wall != nullptr) {
    const uint32_t w4 = __ldg(reinterpret_cast<const unsigned int*>(a.wall + rbase + k));
#pragma unroll
    for (int j = 0; j < 4; ++j) w[j] = ((w4 >> (8 * j)) & 0xffu) != 0;
  }
  if (__any_sync(0xffffffffu, w[0] || w[1] || w[2] || w[3])) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (w[j]) wall_swap<Q>(d[j]);
  }
  Cell x;
  x.i0 = i0;
  x.i1 = i1;
  x.row = rbase;
  x.srow = sbase;
  if constexpr (FACES) {
    bool near = false;
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
      const FaceK& fc = a.face[fi];
      if (fc.kind == kFaceNone) continue;
      const uint32_t ins = a.face_inset;
      if (fc.axis == 0) near |= i0 == (fc.side == 0 ? ins : g.n0 - 1 - ins);
      else if (fc.axis == 1) near |= i1 == (fc.side == 0 ? ins : g.n1 - 1 - ins);
      else near |= (fc.side == 0 ? ins : g.n2 - 1 - ins) - k <= 3u;  // one of k..k+3
    }
    if (near) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (w[j]) continue;
        x.c = rbase + k + j;
        x.k = k + j;
        apply_faces<Q, S>(a, x, d[j]);
      }
    }
  }
  uint32_t seed[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    x.c = rbase + k + j;
    x.k = k + j;
    seed[j] = pair_cell<Q, S, FORCE>(a, x, d[j]);
  }
  if (!store) return;
  S* pout = static_cast<S*>(a.pout);
  const uint32_t s01 = sr_pair(seed[0], seed[1]), s23 = sr_pair(seed[2], seed[3]);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    uint2 w;
    w.x = sr_two<S>(d[0][q], d[1][q], s01);
    w.y = sr_two<S>(d[2][q], d[3][q], s23);
    *reinterpret_cast<uint2*>(pout + (static_cast<uint32_t>(q) * g.pstride + sbase + k)) = w;
  }
}

// Row-segment form: block = W warps = 128 W consecutive cells of one row.
template <int Q, class S, bool FACES, bool FORCE, int W>
__global__ void __launch_bounds__(32 * W, quad_min_warps<Q>() / W)
    k_step_quad(const __grid_constant__ StepArgs a) {
  const Geo& g = a.g;
  const uint32_t row = blockIdx.x;
  const uint32_t i0 = fdiv(row, g.div_n1);
  const uint32_t i1 = row - i0 * g.n1;
  const uint32_t k = blockIdx.y * (128u * W) + 4u * threadIdx.x;
  const uint32_t kprev = (k == 0 ? g.n2 : k) - 2u;       // word holding cell k - 1 (high)
  const uint32_t knext = k + 4u == g.n2 ? 0u : k + 4u;  // word holding cell k + 4 (low)
  const uint32_t i0m = i0 == 0 ? g.n0 - 1 : i0 - 1, i0p = i0 + 1 == g.n0 ? 0u : i0 + 1;
  const uint32_t i1m = i1 == 0 ? g.n1 - 1 : i1 - 1, i1p = i1 + 1 == g.n1 ? 0u : i1 + 1;
  const S* pin = static_cast<const S*>(a.pin);
  float d[4][Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q);
    const uint32_t s0 = c0 > 0 ? i0m : (c0 < 0 ? i0p : i0);
    const uint32_t s1 = c1 > 0 ? i1m : (c1 < 0 ? i1p : i1);
    quad_pull<Q, S>(pin + (static_cast<uint32_t>(q) * g.pstride + (s0 * g.n1 + s1) * g.rstride),
                    q, k, kprev, knext, d);
  }
  quad_finish<Q, S, FACES, FORCE>(a, i0, i1, k, row, d, true);
}

// Instance-wide form for any row length that is a multiple of 4: quads follow
// the linear cell index and each lane finds its own row; the lanes past the
// last quad redo it without storing.
template <int Q, class S, bool FACES, bool FORCE>
__global__ void __launch_bounds__(kBlock, quad_min_warps<Q>() / (kBlock / 32))
    k_step_gquad(const __grid_constant__ StepArgs a) {
  const Geo& g = a.g;
  const uint32_t nquads = g.ncell >> 2;
  const uint32_t qidx = blockIdx.x * kBlock + threadIdx.x;
  const bool valid = qidx < nquads;
  const uint32_t ci = 4u * (valid ? qidx : nquads - 1u);
  const uint32_t row = fdiv(ci, g.div_n2);
  const uint32_t k = ci - row * g.n2;
  const uint32_t i0 = fdiv(row, g.div_n1);
  const uint32_t i1 = row - i0 * g.n1;
  const uint32_t kprev = (k == 0 ? g.n2 : k) - 2u;
  const uint32_t knext = k + 4u == g.n2 ? 0u : k + 4u;
  const uint32_t i0m = i0 == 0 ? g.n0 - 1 : i0 - 1, i0p = i0 + 1 == g.n0 ? 0u : i0 + 1;
  const uint32_t i1m = i1 == 0 ? g.n1 - 1 : i1 - 1, i1p = i1 + 1 == g.n1 ? 0u : i1 + 1;
  const S* pin = static_cast<const S*>(a.pin);
  float d[4][Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q);
    const uint32_t s0 = c0 > 0 ? i0m : (c0 < 0 ? i0p : i0);
    const uint32_t s1 = c1 > 0 ? i1m : (c1 < 0 ? i1p : i1);
    quad_pull<Q, S>(pin + (static_cast<uint32_t>(q) * g.pstride + (s0 * g.n1 + s1) * g.rstride),
                    q, k, kprev, knext, d);
  }
  quad_finish<Q, S, FACES, FORCE>(a, i0, i1, k, row, d, valid);
}

// Pairs of the state planes' index: pair j holds state cells 2j, 2j + 1 (rows
// of even length -- padded ones included -- so a pair never spans two rows).
// Row coordinates and source rows are per lane.  PAD: padded state rows.
template <int Q, class S, bool FACES, bool FORCE, bool PAD>
__device__ __forceinline__ void gpair_step(const StepArgs& a, uint32_t pidx) {
  using PT = PairT<S>;
  using P = typename PT::P;
  const Geo& g = a.g;
  const uint32_t npairs = g.pstride >> 1;
  const bool valid = pidx < npairs;
  const uint32_t ci = 2u * (valid ? pidx : npairs - 1u);
  const uint32_t r = fdiv(ci, g.div_rstride);  // row index
  const uint32_t k = ci - r * g.rstride;
  const uint32_t i0 = fdiv(r, g.div_n1);
  const uint32_t i1 = r - i0 * g.n1;
  const uint32_t srow = r * g.rstride;
  const uint32_t dm0 = i0 == 0 ? (g.n0 - 1) * g.splane : 0u - g.splane;  // i0 - 1
  const uint32_t dp0 = i0 == g.n0 - 1 ? 0u - (g.n0 - 1) * g.splane : g.splane;
  const uint32_t dm1 = i1 == 0 ? (g.n1 - 1) * g.rstride : 0u - g.rstride;  // i1 - 1
  const uint32_t dp1 = i1 == g.n1 - 1 ? 0u - (g.n1 - 1) * g.rstride : g.rstride;
  const uint32_t kprev = (k == 0 ? g.rstride : k) - 2u;
  const uint32_t knext = k + 2 == g.rstride ? 0u : k + 2;
  // addresses relative to this pair in plane 0: q pstride plus the row
  // deltas is never negative (q = 0 has none; q >= 1 adds at least one plane
  // of pstride >= splane + rstride), so it extends as unsigned
  const S* b0 = static_cast<const S*>(a.pin) + (srow + k);
  const int32_t ep = static_cast<int32_t>(kprev) - static_cast<int32_t>(k);
  const int32_t en = static_cast<int32_t>(knext) - static_cast<int32_t>(k);
  P v[Q];
  P e[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q), c2 = Lat<Q>::c2(q);
    uint32_t off = static_cast<uint32_t>(q) * g.pstride;
    if (c0 > 0) off += dm0;
    if (c0 < 0) off += dp0;
    if (c1 > 0) off += dm1;
    if (c1 < 0) off += dp1;
    const S* base = b0 + off;
    v[q] = PT::ld(base);
    if (c2 > 0) e[q] = PT::ld(base + ep);
    if (c2 < 0) e[q] = PT::ld(base + en);
  }
  pair_finish<Q, S, FACES, FORCE, PAD>(a, i0, i1, k, r * g.n2, srow, v, e, valid);
}

template <int Q, class S, bool FACES, bool FORCE>
__global__ void __launch_bounds__(kBlock, kGPairMinWarps / (kBlock / 32))
    k_step_gpair(const __grid_constant__ StepArgs a) {
  gpair_step<Q, S, FACES, FORCE, false>(a, blockIdx.x * kBlock + threadIdx.x);
}

// Batched ensemble, state steps of members with even rows: a tile of
// kBatchTile cells is kBatchTile / 2 pairs, kBatchTile / (2 kBlock) per thread
// (see k_batched_step for the tile walk and SPEC).
template <int Q, class S, int SPEC, bool PAD>
__global__ void __launch_bounds__(kBlock, kGPairMinWarps / (kBlock / 32))
    k_batched_pair(const StepArgs* __restrict__ args, const BatchTile* __restrict__ tiles,
                   uint32_t ntiles, int which) {
#if LBM_BATCH_ARGS_SMEM
  __shared__ StepArgs sa;
  uint32_t cur = 0xffffffffu;
#endif
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BatchTile tile = tiles[t];
#if LBM_BATCH_ARGS_SMEM
    if (tile.inst != cur) {
      __syncthreads();
      stage_args(sa, args[kBatchArgs * tile.inst + which]);
      __syncthreads();
      cur = tile.inst;
    }
#else
    const StepArgs& sa = args[kBatchArgs * tile.inst + which];
#endif
#pragma unroll 1
    for (int j = 0; j < kBatchTile / (2 * kBlock); ++j) {
      const uint32_t pidx = (tile.first >> 1) + j * kBlock + threadIdx.x;
      // whole warps past the member's last pair skip the step; a partial warp
      // runs it with its extra lanes clamped
      if ((((tile.first >> 1) + j * kBlock + (threadIdx.x & ~31u)) << 1) >= sa.g.pstride) break;
      if constexpr (SPEC == 0) {
        const bool faces = sa.face[0].kind != kFaceNone || sa.face[1].kind != kFaceNone;
        const bool force = sa.force_mode != 0;
        if (faces) {
          if (force) gpair_step<Q, S, true, true, PAD>(sa, pidx);
          else gpair_step<Q, S, true, false, PAD>(sa, pidx);
        } else {
          if (force) gpair_step<Q, S, false, true, PAD>(sa, pidx);
          else gpair_step<Q, S, false, false, PAD>(sa, pidx);
        }
      } else {
        gpair_step<Q, S, ((SPEC - 1) & 2) != 0, ((SPEC - 1) & 1) != 0, PAD>(sa, pidx);
      }
    }
  }
}

}  // namespace lbm
