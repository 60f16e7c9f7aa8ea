// Device kernels of the lattice-Boltzmann node step (sm_100a).
//
// Reference algorithm: MADDENING LBMNode.update (src/maddening/nodes/lbm.py:899-986):
//   rho, u   = moments(f) with the Guo half step F/2          (lbm.py:934, 209-239)
//   f*       = f - (f - feq(rho,u))/tau + S_guo(rho,u,F)       (lbm.py:937-939)
//   f_str    = periodic roll of f* by e_q on every axis         (lbm.py:942, 242-267)
//   f_bc     = where(wall, f_str[..., opp], f_str)              (lbm.py:944-948)
//   faces    : inlet then outlet                                (lbm.py:950-968)
//   outputs  = moments(f_bc) with F/2, u = 0 in walls, p = rho cs2 (lbm.py:970-976)
//
// Data layout in HBM: structure of arrays, cells in the reference's C order.
//   plane q (q = 0..Q-1) holds population q of every cell as the normalised
//   offset d_q = (f_q - w_q) / w_q.  The ~1e-3 deviations keep full relative
//   precision in FP32, FP16 and BF16, and the moments become fused
//   multiply-adds with the weights.
// The state between steps holds POST-COLLISION offsets p = C(f).  One pass
// (k_step) reads p at x - e_q (pull), applies the wall swap and the faces
// (this is the reference's f_bc), takes the moments (the reference's
// outputs) and collides again, writing p for the next step: 19 loads and 19
// stores per cell, each warp access one contiguous 32-element run.
//
// One thread owns one cell.  For FP32 storage this beat 2- and 4-cell vector
// forms on B200: the wider forms need more registers than 32 resident warps
// per SM allow, and the lost occupancy costs more than the wider accesses save.
// 16-bit storage moves too few bytes per cell for that: it takes two or four
// cells per thread (lbm_pair.cuh) and rounds stochastically (below).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "lbm_lattice.cuh"

namespace lbm {

// ---------------------------------------------------------------------------
// Storage traits
// ---------------------------------------------------------------------------

template <class S>
struct StoreT {
  using R = float;   // arithmetic type
  using IO = float;  // type of f / force / moment buffers at the ABI
};
template <>
struct StoreT<double> {
  using R = double;
  using IO = double;
};

__device__ __forceinline__ float to_r(float s) { return s; }
__device__ __forceinline__ double to_r(double s) { return s; }
__device__ __forceinline__ float to_r(__half s) { return __half2float(s); }
__device__ __forceinline__ float to_r(__nv_bfloat16 s) { return __bfloat162float(s); }

template <class S>
__device__ __forceinline__ S from_r(typename StoreT<S>::R v);
template <>
__device__ __forceinline__ float from_r<float>(float v) { return v; }
template <>
__device__ __forceinline__ double from_r<double>(double v) { return v; }
// 16-bit storage rounds stochastically (sr_one / sr_two below).

template <class S>
__device__ __forceinline__ typename StoreT<S>::R ld_pop(const S* p) {
  return to_r(__ldg(p));
}

// ---------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------

// x / d for 0 <= x < 2^31 by multiply-high and shift (precomputed on the host).
struct FastDiv {
  uint32_t d, m, s;
};
__device__ __forceinline__ uint32_t fdiv(uint32_t x, const FastDiv& f) {
  return (__umulhi(x, f.m) + x) >> f.s;
}

enum FaceKind : int { kFaceNone = 0, kFacePressure = 1, kFaceVelocity = 2, kFaceZeroGrad = 3 };

struct FaceK {
  int kind;
  int axis;  // internal axis 0..2
  int side;  // 0 = min, 1 = max
  int ref_axis;
  double v[3];  // pressure: v[0] = rho_p; velocity: u in INTERNAL axis order
};

constexpr int kMaxQ = 19;

struct Geo {
  uint32_t n0, n1, n2;  // internal dims, a2 contiguous
  uint32_t plane;       // n1 * n2
  uint32_t ncell;       // n0 * n1 * n2
  FastDiv div_n2, div_n1;
  // Layout of the population planes of the state: row stride, plane stride
  // (n1 rows) and plane size.  Equal to n2, plane, ncell, except for a
  // batched member whose rows are padded to an even length (n2 + 1) so that
  // it can run the paired step; the padding cell of a row is never read.
  // Reference-layout arrays (f in/out, wall, force, moments) stay unpadded.
  uint32_t rstride, splane, pstride;
  FastDiv div_rstride;
};

struct StepArgs {
  Geo g;
  double omega;  // 1 / tau
  double guo_c;  // 1 - 1 / (2 tau)
  int force_mode;
  double force[3];  // uniform force, internal axis order
  const void* force_field;
  const uint8_t* wall;
  FaceK face[2];  // [0] inlet, [1] outlet
  const float* dev_values;
  // State buffers (S): population q of cell c at base[q * ncell + c].  The
  // index is 32-bit (plans keep Q x ncell < 2^32): one wide multiply-add per
  // access forms the address.
  const void* pin;
  void* pout;
  const void* f_in;        // AoS IO (prepare)
  void* f_out;             // AoS IO (final step)
  void* rho;
  void* vel;
  void* prs;
  uint32_t mflags;
  int* status;  // device word; bit 0 set when a bounded wait gave up (staged path)
  // Face planes sit this many cells inside the lattice: 0, or 1 for a
  // halo-padded block (the faces act on the interior).
  uint32_t face_inset;
  // force_mode 3 (the pipe node): x force force[0] on the cells of plane i0 =
  // prop_x where prop_mask[i1 n2 + k] is set, z force force[2] on every
  // non-wall cell; moments without the half-force step.
  uint32_t prop_x;
  const uint8_t* prop_mask;
  // k_step covers cells [cell0, cell_end) of the plan (0 and ncell by default:
  // a runner that steps a block plane range by plane range sets them).
  uint32_t cell0, cell_end;
  // Added to a cell's index where it seeds the stochastic rounding of 16-bit
  // storage, so that a block of a larger lattice rounds as that lattice does.
  uint32_t sr_offset;
};

constexpr uint32_t kMomDensityDev = 1u;
constexpr uint32_t kMomRawVelocity = 2u;  // velocity not zeroed in wall cells

// Uniform force in internal axis order; device-resident values (traced
// scalars, dev_values[6..8]) override the host ones.
template <int Q, class R>
__device__ __forceinline__ void uniform_force(const StepArgs& a, R (&F)[3]) {
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
#pragma unroll
  for (int d = 0; d < 3; ++d) F[d] = static_cast<R>(a.force[d]);
  if (a.dev_values != nullptr && a.force_mode == 1) {
    F[0] = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) F[d + sh] = static_cast<R>(a.dev_values[6 + d]);
  }
}

// Value j (internal axis order for velocities) of face condition fi.
template <int Q>
__device__ __forceinline__ double face_value(const StepArgs& a, int fi, int j) {
  constexpr int sh = 3 - Lat<Q>::D;
  if (a.dev_values == nullptr) return a.face[fi].v[j];
  if (a.face[fi].kind == kFacePressure) return j == 0 ? a.dev_values[3 * fi] : 0.0;
  return j < sh ? 0.0 : a.dev_values[3 * fi + j - sh];
}

// ---------------------------------------------------------------------------
// Cell arithmetic on normalised offsets d_q = (f_q - w_q) / w_q
// ---------------------------------------------------------------------------
//
// Every operation below is explicitly rounded (fma_r / mul_r / add_r / sub_r
// are single IEEE operations that the compiler may not fuse or split), so
// each kernel that inlines this code -- one cell or two cells per thread,
// batched, staged -- produces bit-identical results.

__device__ __forceinline__ float fma_r(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_r(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_r(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_r(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_r(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_r(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_r(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_r(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float div_r(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_r(double a, double b) { return __ddiv_rn(a, b); }
// correctly rounded reciprocal (the same value as div_r(1, x))
__device__ __forceinline__ float rcp_r(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp_r(double x) { return __drcp_rn(x); }

// sum_a s_a x_a over the nonzero components s_a = +-1 of a direction (exact
// sign flips; the additions are rounded in axis order).
template <class R>
__device__ __forceinline__ R dot_e(int e0, int e1, int e2, const R (&x)[3]) {
  R v = 0;
  bool first = true;
  const int e[3] = {e0, e1, e2};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (e[k] == 0) continue;
    const R t = e[k] > 0 ? x[k] : -x[k];
    v = first ? t : add_r(v, t);
    first = false;
  }
  return v;
}

template <class R>
struct Mom {
  R rd;    // rho - 1
  R rho;   // rho
  R u[3];  // velocity (internal axes), includes the Guo F/2 half step
};

// ---------------------------------------------------------------------------
// Stochastic rounding of the 16-bit state
// ---------------------------------------------------------------------------
// Round-to-nearest storage of a slowly changing field drops, the same way every
// step, the part of each step's change that is below half a unit in the last
// place: a body-force-driven flow whose offsets (~4e-3) gain ~8e-6 per step --
// two FP16 units -- drifts by 2e-2 relative L2 in 500 steps.  Stochastic
// rounding (up with probability equal to the dropped fraction of a unit) is
// unbiased and keeps such runs at ~1e-4.  The 16 random bits of population q
// of a cell are a hash of the cell's index and of its moments this step (they
// change whenever the flow does): every kernel form rounds every value alike,
// so the forms stay bit-identical, and CUDA-graph replays need no step counter.
// The conversion is cvt.rs.{f16x2,bf16x2}.f32, whose upper / lower 16 random
// bits drive the upper / lower half (measured on B200: unbiased means, halves
// independent, zero bits truncate).  A value's random bits are the low 16 bits
// of its own FP32 pattern XOR the cell's hash: uniform whatever the value (the
// hash is), without a hash per value.
// Only the low 16 bits of the seed are used: the index and the moments' bits
// are folded together, one multiply spreads every input bit upwards and the
// high half is folded back down.
__device__ __forceinline__ uint32_t sr_seed(uint32_t idx, float u0, float u1, float u2,
                                            float rd) {
  uint32_t x = idx ^ __float_as_uint(u0) ^ __float_as_uint(u1) ^ __float_as_uint(u2) ^
               __float_as_uint(rd);
  x *= 0x9E3779B1u;
  return x ^ (x >> 16);
}

// Random bits of value v of a cell with seed `seed` (the low 16 are used).
__device__ __forceinline__ uint32_t sr_bits(uint32_t seed, float v) {
  return __float_as_uint(v) ^ seed;
}

template <class S>
__device__ __forceinline__ uint32_t cvt_rs2(float hi, float lo, uint32_t rbits);
template <>
__device__ __forceinline__ uint32_t cvt_rs2<__half>(float hi, float lo, uint32_t rbits) {
  uint32_t d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
  return d;
}
template <>
__device__ __forceinline__ uint32_t cvt_rs2<__nv_bfloat16>(float hi, float lo, uint32_t rbits) {
  uint32_t d;
  asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
  return d;
}

// One 16-bit value, stochastically rounded with the low 16 bits of r.
template <class S>
__device__ __forceinline__ S sr_one(float v, uint32_t r) {
  const uint32_t d = cvt_rs2<S>(0.0f, v, r & 0xffffu);
  const unsigned short h = static_cast<unsigned short>(d & 0xffffu);
  return *reinterpret_cast<const S*>(&h);
}

// Two values of two cells packed as (lo in the low half, hi in the high half),
// each rounded with the low 16 bits of its FP32 pattern XOR its cell's seed;
// seed2 = sr_pair(seed_lo, seed_hi), formed once per pair of cells.
__device__ __forceinline__ uint32_t sr_pair(uint32_t seed_lo, uint32_t seed_hi) {
  return __byte_perm(seed_lo, seed_hi, 0x5410);
}
template <class S>
__device__ __forceinline__ uint32_t sr_two(float lo, float hi, uint32_t seed2) {
  return cvt_rs2<S>(hi, lo,
                    __byte_perm(__float_as_uint(lo), __float_as_uint(hi), 0x5410) ^ seed2);
}

// rho = sum f; rho u = sum f e + F/2; u = rho u / max(rho, 1e-10)  (lbm.py:209-239)
// With f = w (1 + d): rho - 1 = sum w d, rho u = sum w e d (+F/2).
//
// The sums use the weights as exact integers, w_q = wr_q / 36 (D3Q19: 12, 2,
// 1; D2Q9: 16, 4, 1), and divide by 36 once, with a split constant (rho - 1)
// or inside the reciprocal (u).  A weight rounded to the arithmetic type
// (1/18, 1/36 are not representable) would rescale the momentum handed to the
// equilibrium by the same factor every step; the collide then injects that
// relative error into the populations each step and it compounds over a
// rollout (FP32: 1.3e-5 relative L2 of u after 500 steps of the 64^3 channel,
// against 2.9e-6 with exact weights).
template <int Q, class R, bool FORCE = true>
__device__ __forceinline__ Mom<R> moments(const R (&d)[Q], const R (&F)[3], bool half = true) {
  constexpr double kDen = Lat<Q>::kWDen;
  R rdp = mul_r(static_cast<R>(Lat<Q>::wr(0)), d[0]);  // 36 (rho - 1)
  R m[3] = {0, 0, 0};                                   // 36 rho u
  bool used[3] = {false, false, false};
#pragma unroll
  for (int q = 1; q < Q; ++q) {
    if (q > Lat<Q>::opp(q)) continue;  // visit each (q, opp) pair once
    const int o = Lat<Q>::opp(q);
    const R w = static_cast<R>(Lat<Q>::wr(q));
    const R s = add_r(d[q], d[o]);
    const R t = sub_r(d[q], d[o]);
    rdp = fma_r(w, s, rdp);
    const int e[3] = {Lat<Q>::c0(q), Lat<Q>::c1(q), Lat<Q>::c2(q)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (e[k] == 0) continue;
      const R ws = e[k] > 0 ? w : -w;
      m[k] = used[k] ? fma_r(ws, t, m[k]) : mul_r(ws, t);
      used[k] = true;
    }
  }
  if constexpr (FORCE) {
    if (half) {
#pragma unroll
      for (int k = 0; k < 3; ++k) m[k] = fma_r(static_cast<R>(0.5 * kDen), F[k], m[k]);
    }
  }
  // 1/36 = c_hi + c_lo to twice the working precision
  constexpr R c_hi = static_cast<R>(1.0 / kDen);
  constexpr R c_lo = static_cast<R>(1.0 / kDen - static_cast<double>(c_hi));
  Mom<R> r;
  r.rd = fma_r(rdp, c_hi, mul_r(rdp, c_lo));
  r.rho = add_r(R(1), r.rd);
  const R den = r.rho > R(1e-10) ? r.rho : R(1e-10);
  const R inv = rcp_r(mul_r(static_cast<R>(kDen), den));  // 1 / (36 rho)
#pragma unroll
  for (int k = 0; k < 3; ++k) r.u[k] = mul_r(m[k], inv);
  return r;
}

// BGK relax towards feq plus the Guo source term (lbm.py:180-206, 307-353,
// 937-939), divided by w_q:
//   deq_q = rho' + rho (3 eu + 4.5 eu^2 - 1.5 u^2)
//   s_q   = (1 - 1/(2 tau)) (3 (e_q - u).F + 9 (e_q.u)(e_q.F))
//   p_q   = d_q - (d_q - deq_q) / tau + s_q
//         = (1 - omega) d_q + A_q + B_q
// with the even part A_q = omega (rho' - 1.5 rho u^2 + 4.5 rho eu^2)
// + c (9 eu eF - 3 u.F) and the odd part B_q = 3 omega rho eu + 3 c eF, so a
// direction and its opposite share A and negate B.  Without a force the
// velocity terms fold into one product, eu (4.5 omega rho eu +- 3 omega rho).
template <int Q, class R, bool FORCE>
__device__ __forceinline__ void collide(R (&d)[Q], const Mom<R>& m, const R (&F)[3], R omega,
                                        R guo_c) {
  const R usq = fma_r(m.u[0], m.u[0], fma_r(m.u[1], m.u[1], mul_r(m.u[2], m.u[2])));
  const R orho = mul_r(omega, m.rho);
  // omega (rho' - 1.5 rho u^2)
  const R base = fma_r(omega, m.rd, mul_r(mul_r(R(-1.5), orho), usq));
  const R r45 = mul_r(R(4.5), orho);
  const R r3 = mul_r(R(3), orho);
  const R keep = sub_r(R(1), omega);
  R c3 = 0, c9 = 0, cuF = 0, even0 = base;
  if constexpr (FORCE) {
    const R uF = fma_r(m.u[0], F[0], fma_r(m.u[1], F[1], mul_r(m.u[2], F[2])));
    c3 = mul_r(R(3), guo_c);
    c9 = mul_r(R(9), guo_c);
    cuF = mul_r(c3, uF);  // c 3 u.F
    even0 = sub_r(base, cuF);
  }
  d[0] = fma_r(keep, d[0], even0);
#pragma unroll
  for (int q = 1; q < Q; ++q) {
    if (q > Lat<Q>::opp(q)) continue;
    const int o = Lat<Q>::opp(q);
    const int e0 = Lat<Q>::c0(q), e1 = Lat<Q>::c1(q), e2 = Lat<Q>::c2(q);
    const R eu = dot_e(e0, e1, e2, m.u);
    const R dq = d[q], dop = d[o];
    if constexpr (FORCE) {
      // c 9 e.F and c 3 e.F depend on the force only: the cells of a thread
      // that share a uniform force share them
      const R eF = dot_e(e0, e1, e2, F);
      const R c9eF = mul_r(c9, eF), c3eF = mul_r(c3, eF);
      R A = fma_r(r45, mul_r(eu, eu), base);
      A = add_r(A, fma_r(eu, c9eF, -cuF));
      const R B = fma_r(r3, eu, c3eF);
      d[q] = add_r(fma_r(keep, dq, A), B);
      d[o] = sub_r(fma_r(keep, dop, A), B);
    } else {
      // (1 - omega) d + base + eu (4.5 omega rho eu +- 3 omega rho)
      d[q] = fma_r(eu, fma_r(r45, eu, r3), fma_r(keep, dq, base));
      d[o] = fma_r(eu, fma_r(r45, eu, -r3), fma_r(keep, dop, base));
    }
  }
}

// Reference Zou-He pressure face (lbm.py:425-510).  Its closure
// u_n = +-(1 - (S_known + S_tang) / rho_p) carries no factor 2 on S_known;
// kept as is.  The known+tangential weights sum to 5/6 on both lattices, so
// u_n = s (rho_p - 5/6 - G) / rho_p with G the sum of their w d.
// Unknown q: f_q = f_opp + feq_q - feq_opp, i.e. d_q = d_opp + 6 rho_p e_qa u_n.
template <int Q, class R>
__device__ __forceinline__ void face_pressure(R (&d)[Q], const StepArgs& a, int fi) {
  const FaceK& fc = a.face[fi];
  const int ax = fc.axis;
  const bool mn = fc.side == 0;
  R G = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (!unknown) G = fma_r(static_cast<R>(Lat<Q>::w(q)), d[q], G);
  }
  const double rho_p = face_value<Q>(a, fi, 0);
  const double rho_c = rho_p > 1e-10 ? rho_p : 1e-10;
  const R c1 = static_cast<R>(rho_c - 5.0 / 6.0);
  R un = div_r(sub_r(c1, G), static_cast<R>(rho_c));
  if (!mn) un = -un;
  const R k6 = mul_r(static_cast<R>(6.0 * rho_p), un);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (unknown) d[q] = cq > 0 ? add_r(d[Lat<Q>::opp(q)], k6) : sub_r(d[Lat<Q>::opp(q)], k6);
  }
}

// Velocity face (extension): rho = (S_tang + 2 S_known) / (1 - s u_a); the
// tangential plus twice the known weights sum to 1, so
// rho = (1 + G) / (1 - s u_a) with G = sum_tang w d + 2 sum_known w d;
// unknown q: d_q = d_opp + 6 rho (e_q . u).
template <int Q, class R>
__device__ __forceinline__ void face_velocity(R (&d)[Q], const StepArgs& a, int fi) {
  const FaceK& fc = a.face[fi];
  const int ax = fc.axis;
  const bool mn = fc.side == 0;
  R G = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    const R w = static_cast<R>(Lat<Q>::w(q));
    if (cq == 0) G = fma_r(w, d[q], G);
    else if (!unknown) G = fma_r(R(2) * w, d[q], G);
  }
  const R uf[3] = {static_cast<R>(face_value<Q>(a, fi, 0)),
                   static_cast<R>(face_value<Q>(a, fi, 1)),
                   static_cast<R>(face_value<Q>(a, fi, 2))};
  const R ua = uf[ax];
  const R rho6 = div_r(mul_r(R(6), add_r(R(1), G)), mn ? sub_r(R(1), ua) : add_r(R(1), ua));
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (unknown) {
      const R eu = dot_e(Lat<Q>::c0(q), Lat<Q>::c1(q), Lat<Q>::c2(q), uf);
      d[q] = fma_r(rho6, eu, d[Lat<Q>::opp(q)]);
    }
  }
}

__device__ __forceinline__ uint32_t wrapu(int i, uint32_t n) {
  return static_cast<uint32_t>(i < 0 ? i + static_cast<int>(n)
                                     : (i >= static_cast<int>(n) ? i - static_cast<int>(n) : i));
}

// The value of population q that the reference's f_bc holds at cell
// (i0,i1,k): the pulled p[x - e_q] or, in a wall cell, p[x + e_q] of opp(q).
template <int Q, class S>
__device__ __forceinline__ typename StoreT<S>::R fbc_at(const StepArgs& a, int q, int i0,
                                                        int i1, int k) {
  const Geo& g = a.g;
  const bool wl =
      a.wall != nullptr && a.wall[(static_cast<uint32_t>(i0) * g.n1 + i1) * g.n2 + k] != 0;
  const int s = wl ? 1 : -1;
  const int qs = wl ? Lat<Q>::opp(q) : q;
  const uint32_t j0 = wrapu(i0 + s * Lat<Q>::c0(q), g.n0);
  const uint32_t j1 = wrapu(i1 + s * Lat<Q>::c1(q), g.n1);
  const uint32_t j2 = wrapu(k + s * Lat<Q>::c2(q), g.n2);
  return ld_pop<S>(static_cast<const S*>(a.pin) +
                   (static_cast<uint32_t>(qs) * g.pstride + (j0 * g.n1 + j1) * g.rstride + j2));
}

// Zero-gradient face (extension): unknown q <- f_bc of the neighbour one
// cell inwards (its post-stream, post-bounce value).
template <int Q, class S>
__device__ __forceinline__ void face_zero_gradient(typename StoreT<S>::R (&d)[Q], const StepArgs& a,
                                                int fi, int i0, int i1, int k) {
  const FaceK& fc = a.face[fi];
  const int ax = fc.axis;
  const bool mn = fc.side == 0;
  const int st = mn ? 1 : -1;
  const int n0 = i0 + (ax == 0 ? st : 0), n1 = i1 + (ax == 1 ? st : 0), n2 = k + (ax == 2 ? st : 0);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (unknown) d[q] = fbc_at<Q, S>(a, q, n0, n1, n2);
  }
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Launch shape of the step kernels: 128 threads, >= 10 blocks per SM (<= 51
// registers, 40 resident warps); the fastest shape of a B200 sweep.
#ifndef LBM_STEP_BLOCK
#define LBM_STEP_BLOCK 128
#endif
#ifndef LBM_STEP_MINB
#define LBM_STEP_MINB 10
#endif
constexpr int kBlock = LBM_STEP_BLOCK;
constexpr int kMinBlocks = LBM_STEP_MINB;
// FP64 arithmetic holds twice the registers: half the resident blocks.
template <class S>
constexpr int min_blocks() { return sizeof(typename StoreT<S>::R) == 8 ? kMinBlocks / 2 : kMinBlocks; }
// The batched kernels also hold a member's arguments: 8 blocks (64 registers).
template <class S>
constexpr int batched_min_blocks() { return sizeof(typename StoreT<S>::R) == 8 ? 4 : 8; }

// kOutState: the next state; kOutAoS: the reference f (last step); kOutMoments:
// moments only; kOutRecord: the next state and, where the pointers are set,
// the reference f and the moments of this step (a recorded history step).
enum StepMode : int { kOutState = 0, kOutAoS = 1, kOutMoments = 2, kOutRecord = 3 };

// ---------------------------------------------------------------------------
// Block-staged stores to the reference layout (*grid, Q)
// ---------------------------------------------------------------------------
// The kBlock cells of a block are consecutive, so their Q values each form one
// contiguous run of the output.  Written directly, thread t's values sit Q
// elements apart from thread t+1's and every store instruction of a warp
// touches 32 separate sectors; staged here, the block writes the run with
// 16-byte stores.  Thread t of the block owns row t of the tile.
template <int Q, class IO>
__device__ __forceinline__ IO* aos_tile() {
  __shared__ __align__(16) IO tile[kBlock * Q];
  return tile;
}

// Writes the tile rows of cells [first, min(first + kBlock, ncell)) to
// out[first * Q ...].  Every thread of the block must call it (it holds the
// barriers on both sides, so the tile can be refilled afterwards).
template <int Q, class IO>
__device__ __forceinline__ void aos_flush(IO* out, uint32_t first, uint32_t ncell) {
  const IO* tile = aos_tile<Q, IO>();
  __syncthreads();
  if (first < ncell) {
    const uint32_t cells = ncell - first < static_cast<uint32_t>(kBlock) ? ncell - first : kBlock;
    const uint32_t n = cells * Q;
    IO* dst = out + static_cast<size_t>(first) * Q;
    uint32_t done = 0;
    if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
      constexpr uint32_t V = 16 / sizeof(IO);
      const uint32_t nv = n / V;
      const uint4* src4 = reinterpret_cast<const uint4*>(tile);
      uint4* dst4 = reinterpret_cast<uint4*>(dst);
      for (uint32_t i = threadIdx.x; i < nv; i += kBlock) dst4[i] = src4[i];
      done = nv * V;
    }
    for (uint32_t i = done + threadIdx.x; i < n; i += kBlock) dst[i] = tile[i];
  }
  __syncthreads();
}

// Reads the values of cells [first, min(first + kBlock, ncell)) from
// in[first * Q ...] into the tile (16-byte loads when aligned); afterwards
// thread t finds its cell's Q values in tile row t.  Every thread of the
// block must call it.
template <int Q, class IO>
__device__ __forceinline__ const IO* aos_fill(const IO* in, uint32_t first, uint32_t ncell) {
  IO* tile = aos_tile<Q, IO>();
  __syncthreads();  // an earlier use of the tile is over
  if (first < ncell) {
    const uint32_t cells = ncell - first < static_cast<uint32_t>(kBlock) ? ncell - first : kBlock;
    const uint32_t n = cells * Q;
    const IO* src = in + static_cast<size_t>(first) * Q;
    uint32_t done = 0;
    if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
      constexpr uint32_t V = 16 / sizeof(IO);
      const uint32_t nv = n / V;
      const uint4* src4 = reinterpret_cast<const uint4*>(src);
      uint4* dst4 = reinterpret_cast<uint4*>(tile);
      for (uint32_t i = threadIdx.x; i < nv; i += kBlock) dst4[i] = __ldg(src4 + i);
      done = nv * V;
    }
    for (uint32_t i = done + threadIdx.x; i < n; i += kBlock) tile[i] = __ldg(src + i);
  }
  __syncthreads();
  return tile + threadIdx.x * Q;
}

struct Cell {
  uint32_t c;      // linear cell index (reference layout)
  uint32_t i0, i1, k;
  uint32_t row;    // c - k
  uint32_t srow;   // start of the row in the state planes
};

__device__ __forceinline__ Cell locate(const Geo& g, uint32_t c) {
  Cell x;
  x.c = c;
  const uint32_t r = fdiv(c, g.div_n2);  // row index
  x.k = c - r * g.n2;
  x.i0 = fdiv(r, g.div_n1);
  x.i1 = r - x.i0 * g.n1;
  x.row = c - x.k;
  x.srow = r * g.rstride;
  return x;
}

// The index whose hash seeds the stochastic rounding of cell x: its reference-
// layout index; in a halo-padded block (face_inset = 1) the periodic index of
// the interior lattice, so that a periodic pad rounds as the unpadded lattice.
template <int Q>
__device__ __forceinline__ uint32_t sr_index(const StepArgs& a, const Cell& x) {
  if (a.face_inset == 0) return x.c + a.sr_offset;
  const Geo& g = a.g;
  auto in = [](uint32_t i, uint32_t n) { return i == 0 ? n - 3 : (i + 1 == n ? 0u : i - 1); };
  const uint32_t j0 = Lat<Q>::D == 3 ? in(x.i0, g.n0) : 0u;
  return (j0 * (g.n1 - 2) + in(x.i1, g.n1)) * (g.n2 - 2) + in(x.k, g.n2);
}

// Pipe-node force of cell c (force_mode 3, LBMPipeNode.update lbm_pipe.py:766-779).
template <class R>
__device__ __forceinline__ void pipe_force(const StepArgs& a, uint32_t c, bool wall, R (&F)[3]) {
  const Geo& g = a.g;
  const uint32_t r = fdiv(c, g.div_n2);
  const uint32_t k = c - r * g.n2;
  const uint32_t i0 = fdiv(r, g.div_n1);
  const uint32_t i1 = r - i0 * g.n1;
  F[0] = (i0 == a.prop_x && __ldg(a.prop_mask + i1 * g.n2 + k) != 0) ? static_cast<R>(a.force[0])
                                                                        : R(0);
  F[1] = 0;
  F[2] = wall ? R(0) : static_cast<R>(a.force[2]);
}

template <int Q, class IO>
__device__ __forceinline__ void load_force(const void* force_field, uint32_t c,
                                           typename StoreT<IO>::R (&F)[3]) {
  using R = typename StoreT<IO>::R;
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  const IO* p = static_cast<const IO*>(force_field) + static_cast<size_t>(c) * D;
  F[0] = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) F[d + sh] = static_cast<R>(__ldg(p + d));
}

template <int Q, class IO>
__device__ __forceinline__ void store_moments(const StepArgs& a, uint32_t c,
                                              const Mom<typename StoreT<IO>::R>& m, bool wall) {
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  if (a.rho != nullptr)
    static_cast<IO*>(a.rho)[c] = (a.mflags & kMomDensityDev) ? m.rd : m.rho;
  if (a.prs != nullptr) {
    if constexpr (sizeof(IO) == 8) static_cast<IO*>(a.prs)[c] = mul_r(m.rho, 1.0 / 3.0);
    else static_cast<IO*>(a.prs)[c] = mul_r(m.rho, static_cast<float>(1.0 / 3.0));
  }
  if (a.vel != nullptr) {
    IO* v = static_cast<IO*>(a.vel) + static_cast<size_t>(c) * D;
    const bool zero = wall && !(a.mflags & kMomRawVelocity);
#pragma unroll
    for (int d = 0; d < D; ++d) v[d] = zero ? IO(0) : static_cast<IO>(m.u[d + sh]);
  }
}

// Reference state f (IO) -> normalised offset, and back.  The offset
// d = (f - w_q) / w_q = f (1 / w_q) - 1 is one fused multiply-add: 1 / w_q is
// an integer or a short binary fraction (D3Q19: 3, 18, 36; D2Q9: 2.25, 9,
// 36), exact in float and double, so the FMA forms f / w_q - 1 exactly and
// rounds it once.
template <int Q, class R>
__device__ __forceinline__ R to_offset(R f, int q) {
  return fma_r(f, static_cast<R>(static_cast<double>(Lat<Q>::kWDen) / Lat<Q>::wr(q)), R(-1));
}
template <int Q, class R>
__device__ __forceinline__ R from_offset(R d, int q) {
  if constexpr (sizeof(R) == 8) return fma_r(Lat<Q>::w(q), d, Lat<Q>::w(q));
  else return add_r(w_hi<Q>(q), fma_r(w_hi<Q>(q), d, w_lo<Q>(q)));
}

// Collide from a reference-layout state f (*grid_shape, Q): p = C(f).
// Cell-local; the first pass of every update / rollout.
// fi: the cell's Q reference values (a tile row filled by aos_fill).
template <int Q, class S, bool FORCE>
__device__ __forceinline__ void prepare_cell(const StepArgs& a, uint32_t c,
                                             const typename StoreT<S>::IO* fi) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  // index in the state planes (differs only for padded rows)
  const uint32_t ci =
      a.g.rstride == a.g.n2 ? c : c + fdiv(c, a.g.div_n2) * (a.g.rstride - a.g.n2);
  R d[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) d[q] = to_offset<Q, R>(static_cast<R>(fi[q]), q);
  R F[3] = {0, 0, 0};
  if (FORCE) {
    if (a.force_mode == 2) load_force<Q, IO>(a.force_field, c, F);
    else if (a.force_mode == 3) pipe_force<R>(a, c, a.wall != nullptr && a.wall[c] != 0, F);
    else uniform_force<Q, R>(a, F);
  }
  const Mom<R> m = moments<Q, R, FORCE>(d, F, a.force_mode != 3);
  if (a.rho != nullptr || a.vel != nullptr || a.prs != nullptr)
    store_moments<Q, IO>(a, c, m, a.wall != nullptr && a.wall[c] != 0);
  collide<Q, R, FORCE>(d, m, F, static_cast<R>(a.omega), static_cast<R>(a.guo_c));
  if constexpr (sizeof(S) == 2) {
    Cell x;
    if (a.face_inset != 0) x = locate(a.g, c);
    else x.c = c;
    const uint32_t seed = sr_seed(sr_index<Q>(a, x), m.u[0], m.u[1], m.u[2], m.rd);
#pragma unroll
    for (int q = 0; q < Q; ++q)
      static_cast<S*>(a.pout)[static_cast<uint32_t>(q) * a.g.pstride + ci] =
          sr_one<S>(d[q], sr_bits(seed, d[q]));
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q)
      static_cast<S*>(a.pout)[static_cast<uint32_t>(q) * a.g.pstride + ci] = from_r<S>(d[q]);
  }
}

template <int Q, class S, bool FORCE>
__global__ void __launch_bounds__(kBlock, min_blocks<S>())
    k_prepare(const __grid_constant__ StepArgs a) {
  using IO = typename StoreT<S>::IO;
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  const IO* row = aos_fill<Q, IO>(static_cast<const IO*>(a.f_in), blockIdx.x * kBlock, a.g.ncell);
  if (c < a.g.ncell) prepare_cell<Q, S, FORCE>(a, c, row);
}

// Wall-node swap (lbm.py:944-948): a wall cell takes f_str[..., opp].
template <int Q, class R>
__device__ __forceinline__ void wall_swap(R (&d)[Q]) {
#pragma unroll
  for (int q = 1; q < Q; ++q) {
    if (q < Lat<Q>::opp(q)) {
      const R t = d[q];
      d[q] = d[Lat<Q>::opp(q)];
      d[Lat<Q>::opp(q)] = t;
    }
  }
}

// Faces of a non-wall cell: inlet first, then outlet (lbm.py:950-968).
template <int Q, class S>
__device__ __forceinline__ void apply_faces(const StepArgs& a, const Cell& x,
                                            typename StoreT<S>::R (&d)[Q]) {
  using R = typename StoreT<S>::R;
  const Geo& g = a.g;
#pragma unroll
  for (int fi = 0; fi < 2; ++fi) {
    const FaceK& fc = a.face[fi];
    if (fc.kind == kFaceNone) continue;
    const uint32_t coord = fc.axis == 0 ? x.i0 : (fc.axis == 1 ? x.i1 : x.k);
    const uint32_t nax = fc.axis == 0 ? g.n0 : (fc.axis == 1 ? g.n1 : g.n2);
    if (coord != (fc.side == 0 ? a.face_inset : nax - 1 - a.face_inset)) continue;
    if (fc.kind == kFacePressure) face_pressure<Q, R>(d, a, fi);
    else if (fc.kind == kFaceVelocity) face_velocity<Q, R>(d, a, fi);
    else face_zero_gradient<Q, S>(d, a, fi, x.i0, x.i1, x.k);
  }
}

// Wall-node swap and faces of one cell's pulled populations: afterwards d is
// the reference's f_bc at that cell.
template <int Q, class S, bool FACES>
__device__ __forceinline__ void apply_bc(const StepArgs& a, const Cell& x, bool wall,
                                         typename StoreT<S>::R (&d)[Q]) {
  // Obstacles are clustered: most warps hold no wall cell and skip the swap.
  if (__any_sync(__activemask(), wall)) {
    if (wall) wall_swap<Q>(d);
  }
  // wall face cells keep the swapped populations
  if constexpr (FACES) {
    if (!wall) apply_faces<Q, S>(a, x, d);
  }
}

// Everything of one fused step after the pull (d = the pulled populations of
// cell x): wall swap -> faces (= reference f_bc) -> moments (reference
// outputs) -> collide (next p), or write f_bc (MODE kOutAoS), or moments only
// (MODE kOutMoments).
template <int Q, class S, int MODE, bool FACES, bool FORCE>
__device__ __forceinline__ void finish_cell(const StepArgs& a, const Cell& x,
                                            typename StoreT<S>::R (&d)[Q]) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  const Geo& g = a.g;
  const uint32_t cidx = x.c;
  const bool wall = a.wall != nullptr && __ldg(a.wall + cidx) != 0;
  R F[3] = {0, 0, 0};
  if (FORCE) {
    if (a.force_mode == 2) load_force<Q, IO>(a.force_field, cidx, F);
    else if (a.force_mode == 3) pipe_force<R>(a, cidx, wall, F);
    else uniform_force<Q, R>(a, F);
  }
  apply_bc<Q, S, FACES>(a, x, wall, d);
  const Mom<R> m = moments<Q, R, FORCE>(d, F, a.force_mode != 3);
  store_moments<Q, IO>(a, cidx, m, wall);

  if constexpr (MODE == kOutAoS || MODE == kOutRecord) {
    // f_bc into this thread's tile row; the kernel writes the block's run
    if (MODE == kOutAoS || a.f_out != nullptr) {
      IO* row = aos_tile<Q, IO>() + threadIdx.x * Q;
#pragma unroll
      for (int q = 0; q < Q; ++q) row[q] = static_cast<IO>(from_offset<Q, R>(d[q], q));
    }
  }
  if constexpr (MODE == kOutState || MODE == kOutRecord) {
    collide<Q, R, FORCE>(d, m, F, static_cast<R>(a.omega), static_cast<R>(a.guo_c));
    if constexpr (sizeof(S) == 2) {
      const uint32_t seed = sr_seed(sr_index<Q>(a, x), m.u[0], m.u[1], m.u[2], m.rd);
#pragma unroll
      for (int q = 0; q < Q; ++q)
        static_cast<S*>(a.pout)[static_cast<uint32_t>(q) * g.pstride + x.srow + x.k] =
            sr_one<S>(d[q], sr_bits(seed, d[q]));
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q)
        static_cast<S*>(a.pout)[static_cast<uint32_t>(q) * g.pstride + x.srow + x.k] =
            from_r<S>(d[q]);
    }
  }
}

// The pulled populations p(x - e_q) of cell x (periodic on every axis).
template <int Q, class S>
__device__ __forceinline__ void pull_cell(const StepArgs& a, const Cell& x,
                                          typename StoreT<S>::R (&d)[Q]) {
  const Geo& g = a.g;
  // Offsets of the source rows of the pull x - e_q (periodic on every axis).
  const uint32_t dm0 = x.i0 == 0 ? (g.n0 - 1) * g.splane : 0u - g.splane;  // i0 - 1
  const uint32_t dp0 = x.i0 == g.n0 - 1 ? 0u - (g.n0 - 1) * g.splane : g.splane;
  const uint32_t dm1 = x.i1 == 0 ? (g.n1 - 1) * g.rstride : 0u - g.rstride;  // i1 - 1
  const uint32_t dp1 = x.i1 == g.n1 - 1 ? 0u - (g.n1 - 1) * g.rstride : g.rstride;
  const uint32_t km = x.k == 0 ? g.n2 - 1 : x.k - 1;
  const uint32_t kp = x.k == g.n2 - 1 ? 0 : x.k + 1;

#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q), c2 = Lat<Q>::c2(q);
    uint32_t off = x.srow;
    if (c0 > 0) off += dm0;
    if (c0 < 0) off += dp0;
    if (c1 > 0) off += dm1;
    if (c1 < 0) off += dp1;
    off += c2 > 0 ? km : (c2 < 0 ? kp : x.k);
    d[q] = ld_pop<S>(static_cast<const S*>(a.pin) + (static_cast<uint32_t>(q) * g.pstride + off));
  }
}

// One fused step of cell cidx: pull p from global memory, then finish_cell.
template <int Q, class S, int MODE, bool FACES, bool FORCE>
__device__ __forceinline__ void step_cell(const StepArgs& a, uint32_t cidx) {
  using R = typename StoreT<S>::R;
  const Cell x = locate(a.g, cidx);
  R d[Q];
  pull_cell<Q, S>(a, x, d);
  finish_cell<Q, S, MODE, FACES, FORCE>(a, x, d);
}

template <int Q, class S, int MODE, bool FACES, bool FORCE>
__global__ void __launch_bounds__(kBlock, min_blocks<S>())
    k_step(const __grid_constant__ StepArgs a) {
  using IO = typename StoreT<S>::IO;
  const uint32_t first = a.cell0 + blockIdx.x * kBlock;
  const uint32_t cidx = first + threadIdx.x;
  if (cidx < a.cell_end) step_cell<Q, S, MODE, FACES, FORCE>(a, cidx);
  if constexpr (MODE == kOutAoS || MODE == kOutRecord) {
    if (MODE == kOutAoS || a.f_out != nullptr)
      aos_flush<Q, IO>(static_cast<IO*>(a.f_out), first, a.cell_end);
  }
}

// Halo-padded block (the reference's update_padded, lbm.py:747-897): one halo
// cell on every side of every spatial axis.  p (the whole block collided) is
// pulled across the halo without wrapping -- interior cells never reach past
// the halo -- then wall swap, faces on the interior planes (face_inset = 1),
// moments and f_bc of the interior cells are written; a halo cell keeps its
// input populations (f_in copied to f_out) and its moment outputs untouched.
template <int Q, class S, bool FACES, bool FORCE>
__global__ void __launch_bounds__(kBlock, min_blocks<S>())
    k_step_padded(const __grid_constant__ StepArgs a) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  const Geo& g = a.g;
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  if (c < g.ncell) {
    const Cell x = locate(g, c);
    const bool halo = (Lat<Q>::D == 3 && (x.i0 == 0 || x.i0 == g.n0 - 1)) || x.i1 == 0 ||
                      x.i1 == g.n1 - 1 || x.k == 0 || x.k == g.n2 - 1;
    if (halo) {
      const IO* fi = static_cast<const IO*>(a.f_in) + static_cast<size_t>(c) * Q;
      IO* row = aos_tile<Q, IO>() + threadIdx.x * Q;
#pragma unroll
      for (int q = 0; q < Q; ++q) row[q] = fi[q];
    } else {
      R d[Q];
      pull_cell<Q, S>(a, x, d);
      finish_cell<Q, S, kOutAoS, FACES, FORCE>(a, x, d);
    }
  }
  aos_flush<Q, IO>(static_cast<IO*>(a.f_out), blockIdx.x * kBlock, g.ncell);
}

// ---------------------------------------------------------------------------
// Batched ensemble: many lattices (own shape, tau, force, walls) in one launch
// ---------------------------------------------------------------------------

// A tile is kBatchTile consecutive cells of one instance (a multiple of
// 2 kBlock: the paired kernel gives each thread kBatchTile / (2 kBlock) pairs).
// 512 cells: on the 64-lattice ensemble 37.4k (FP32) and 54.8k (FP16) MLUPS
// against 36.7k / 52.6k for 256-cell tiles, 36.6k / 55.0k for 1024 and
// 36.0k / 53.1k for 2048 (B200).
#ifndef LBM_BATCH_TILE
#define LBM_BATCH_TILE (4 * LBM_STEP_BLOCK)
#endif
constexpr int kBatchTile = LBM_BATCH_TILE;
static_assert(kBatchTile % (2 * kBlock) == 0, "batch tiles hold whole pair rows of a block");
struct BatchTile {
  uint32_t inst;
  uint32_t first;
};

// Argument blocks per instance: [0] p in B -> out A (also the first collide),
// [1] p in A -> out B, [2] the last step (reference f and moments out).
constexpr int kBatchArgs = 3;

// Per-instance arguments of a batched tile: staged in shared memory (1), or
// read from global memory through the L1 (0).
#ifndef LBM_BATCH_ARGS_SMEM
#define LBM_BATCH_ARGS_SMEM 0
#endif

// Copies instance arguments into shared memory (the whole block reads them).
__device__ __forceinline__ void stage_args(StepArgs& dst, const StepArgs& src) {
  static_assert(sizeof(StepArgs) % 4 == 0, "StepArgs is copied as 32-bit words");
  const uint32_t* s = reinterpret_cast<const uint32_t*>(&src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
  for (int w = threadIdx.x; w < static_cast<int>(sizeof(StepArgs) / 4); w += kBlock) d[w] = s[w];
}

// The face / force specialisation of a member is chosen per tile at run time,
// so every member runs exactly the kernel body its own rollout would.
template <int Q, class S, int MODE>
__device__ __forceinline__ void step_cell_any(const StepArgs& a, uint32_t c) {
  const bool faces = a.face[0].kind != kFaceNone || a.face[1].kind != kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) {
    if (force) step_cell<Q, S, MODE, true, true>(a, c);
    else step_cell<Q, S, MODE, true, false>(a, c);
  } else {
    if (force) step_cell<Q, S, MODE, false, true>(a, c);
    else step_cell<Q, S, MODE, false, false>(a, c);
  }
}

// Persistent launch: each block walks the tile list with a grid stride; tile
// t uses args[kBatchArgs * inst + which], staged in shared memory.  SPEC = 0:
// every member's face / force specialisation is chosen per tile at run time;
// otherwise all members share the one given at compile time (SPEC = 1 +
// 2 FACES + FORCE), which keeps a single copy of the step body in the kernel.
template <int Q, class S, int MODE, int SPEC>
__global__ void __launch_bounds__(kBlock, batched_min_blocks<S>())
    k_batched_step(const StepArgs* __restrict__ args, const BatchTile* __restrict__ tiles,
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
    for (int j = 0; j < kBatchTile / kBlock; ++j) {
      const uint32_t first = tile.first + j * kBlock;  // block-uniform
      if (first >= sa.g.ncell) break;
      const uint32_t c = first + threadIdx.x;
      if (c < sa.g.ncell) {
        if constexpr (SPEC == 0) step_cell_any<Q, S, MODE>(sa, c);
        else step_cell<Q, S, MODE, ((SPEC - 1) & 2) != 0, ((SPEC - 1) & 1) != 0>(sa, c);
      }
      if constexpr (MODE == kOutAoS)
        aos_flush<Q, typename StoreT<S>::IO>(static_cast<typename StoreT<S>::IO*>(sa.f_out),
                                             first, sa.g.ncell);
    }
  }
}

template <int Q, class S>
__global__ void __launch_bounds__(kBlock, batched_min_blocks<S>())
    k_batched_prepare(const StepArgs* __restrict__ args, const BatchTile* __restrict__ tiles,
                      uint32_t ntiles) {
  __shared__ StepArgs sa;
  uint32_t cur = 0xffffffffu;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const BatchTile tile = tiles[t];
    if (tile.inst != cur) {
      __syncthreads();
      stage_args(sa, args[kBatchArgs * tile.inst]);
      __syncthreads();
      cur = tile.inst;
    }
#pragma unroll 1
    for (int j = 0; j < kBatchTile / kBlock; ++j) {
      const uint32_t first = tile.first + j * kBlock;  // block-uniform
      if (first >= sa.g.ncell) break;
      const uint32_t c = first + threadIdx.x;
      using IO = typename StoreT<S>::IO;
      const IO* row = aos_fill<Q, IO>(static_cast<const IO*>(sa.f_in), first, sa.g.ncell);
      if (c < sa.g.ncell) {
        if (sa.force_mode != 0) prepare_cell<Q, S, true>(sa, c, row);
        else prepare_cell<Q, S, false>(sa, c, row);
      }
    }
  }
}

// f = feq(rho, u) in the reference layout (lbm.py:180-206, 719-745).
template <int Q, class IO>
__global__ void __launch_bounds__(kBlock) k_equilibrium(Geo g, const IO* rho, const IO* u, IO* f) {
  using R = typename StoreT<IO>::R;
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  if (c >= g.ncell) return;
  Mom<R> m;
  m.rho = rho ? static_cast<R>(rho[c]) : R(1);
  m.rd = m.rho - R(1);
  m.u[0] = m.u[1] = m.u[2] = 0;
  if (u)
    for (int d = 0; d < D; ++d) m.u[d + sh] = static_cast<R>(u[static_cast<size_t>(c) * D + d]);
  R dq[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) dq[q] = 0;
  const R F[3] = {0, 0, 0};
  collide<Q, R, false>(dq, m, F, R(1), R(0));  // omega = 1: p = deq exactly
#pragma unroll
  for (int q = 0; q < Q; ++q) f[static_cast<size_t>(c) * Q + q] = from_offset<Q, R>(dq[q], q);
}

// FP64 mass / momentum partial sums: block b writes part[4 b .. 4 b + 3].
// Both reduction kernels run with exactly kReduceThreads threads.
constexpr int kReduceThreads = 256;

template <int Q, class IO>
__global__ void __launch_bounds__(kReduceThreads) k_mass_momentum_part(Geo g, const IO* f,
                                                                       double* part) {
  double acc[4] = {0, 0, 0, 0};
  for (size_t cell = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; cell < g.ncell;
       cell += static_cast<size_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double v = static_cast<double>(f[cell * Q + q]) - Lat<Q>::w(q);
      acc[0] += v;
      acc[1] += Lat<Q>::c0(q) * v;
      acc[2] += Lat<Q>::c1(q) * v;
      acc[3] += Lat<Q>::c2(q) * v;
    }
  }
  __shared__ double red[kReduceThreads / 32][4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double v = acc[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int wi = 0; wi < kReduceThreads / 32; ++wi) v += red[wi][threadIdx.x];
    part[4 * blockIdx.x + threadIdx.x] = v;
  }
}

// Final fixed-order reduction of nparts partials; out = {mass, momentum (ref order)}.
template <int Q>
__global__ void __launch_bounds__(kReduceThreads) k_mass_momentum_final(const double* part, int nparts,
                                                             double ncell, double* out) {
  __shared__ double red[kReduceThreads / 32][4];
  double acc[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < nparts; i += blockDim.x)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += part[4 * i + c];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double v = acc[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][c] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[4] = {0, 0, 0, 0};
    for (int wi = 0; wi < kReduceThreads / 32; ++wi)
      for (int c = 0; c < 4; ++c) s[c] += red[wi][c];
    constexpr int D = Lat<Q>::D;
    out[0] = ncell + s[0];
    for (int d = 0; d < D; ++d) out[1 + d] = s[1 + d + (3 - D)];
    for (int d = D; d < 3; ++d) out[1 + d] = 0.0;
  }
}

}  // namespace lbm
