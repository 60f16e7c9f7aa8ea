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
// Data layout in HBM (all structure-of-arrays, cells in the reference's C order):
//   state[q * ncell + cell]  population q of every cell, stored as the offset
//                            g_q = f_q - w_q (F16/BF16: g_q / w_q), so FP32 keeps
//                            the ~1e-3 deviations at full relative precision.
// The state between steps holds POST-COLLISION offsets p = C(f).  One pass
// (k_step) then reads p at x - e_q (pull), applies the wall swap and the faces
// (this is the reference's f_bc), takes the moments (the reference's outputs),
// and collides again, writing p for the next step: 19 loads + 19 stores per cell.
//
// Thread mapping: one thread owns V consecutive cells of a row along the
// contiguous axis a2 (V = 4 for 32-bit and 16-bit storage, 2 for FP64), so
// every population is read and written as one aligned vector.  The one value
// a shifted direction needs from the neighbouring vector comes from the
// adjacent lane by warp shuffle; only lanes at a row or warp edge load it.
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
struct StoreT;
// Cells per thread on the step path, per storage form.  One cell per thread
// at 128 threads x 8 blocks per SM (<= 64 registers, 32 warps resident)
// measured fastest on B200 for every form; wider forms need more registers
// than a full SM of warps can hold.
#ifndef LBM_F32_VEC
#define LBM_F32_VEC 1
#endif
#ifndef LBM_F16_VEC
#define LBM_F16_VEC 1
#endif
#ifndef LBM_F64_VEC
#define LBM_F64_VEC 1
#endif
template <>
struct StoreT<float> {
  using R = float;   // arithmetic type
  using IO = float;  // type of f / force / moment buffers at the ABI
  static constexpr int V = LBM_F32_VEC;
  static constexpr bool kScaled = false;
};
template <>
struct StoreT<__half> {
  using R = float;
  using IO = float;
  static constexpr int V = LBM_F16_VEC;
  static constexpr bool kScaled = true;
};
template <>
struct StoreT<__nv_bfloat16> {
  using R = float;
  using IO = float;
  static constexpr int V = LBM_F16_VEC;
  static constexpr bool kScaled = true;
};
template <>
struct StoreT<double> {
  using R = double;
  using IO = double;
  static constexpr int V = LBM_F64_VEC;
  static constexpr bool kScaled = false;
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
template <>
__device__ __forceinline__ __half from_r<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_r<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}

// Scalar read-only load of one stored element, converted to the arithmetic type.
template <class S>
__device__ __forceinline__ typename StoreT<S>::R ld1(const S* p) {
  return to_r(__ldg(p));
}

// Aligned vector load / store of V stored elements.
template <class S, int V>
struct VIO {
  using R = typename StoreT<S>::R;
  __device__ __forceinline__ static void ld(const S* p, R (&o)[V]) {
#pragma unroll
    for (int r = 0; r < V; ++r) o[r] = to_r(__ldg(p + r));
  }
  __device__ __forceinline__ static void st(S* p, const R (&v)[V]) {
#pragma unroll
    for (int r = 0; r < V; ++r) p[r] = from_r<S>(v[r]);
  }
};
template <>
struct VIO<float, 4> {
  __device__ __forceinline__ static void ld(const float* p, float (&o)[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  __device__ __forceinline__ static void st(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <>
struct VIO<float, 2> {
  __device__ __forceinline__ static void ld(const float* p, float (&o)[2]) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    o[0] = v.x; o[1] = v.y;
  }
  __device__ __forceinline__ static void st(float* p, const float (&v)[2]) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  }
};
template <>
struct VIO<double, 2> {
  __device__ __forceinline__ static void ld(const double* p, double (&o)[2]) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = v.x; o[1] = v.y;
  }
  __device__ __forceinline__ static void st(double* p, const double (&v)[2]) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  }
};
template <>
struct VIO<__half, 4> {
  __device__ __forceinline__ static void ld(const __half* p, float (&o)[4]) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  }
  __device__ __forceinline__ static void st(__half* p, const float (&v)[4]) {
    __half2 a = __floats2half2_rn(v[0], v[1]);
    __half2 b = __floats2half2_rn(v[2], v[3]);
    uint2 u;
    u.x = *reinterpret_cast<uint32_t*>(&a);
    u.y = *reinterpret_cast<uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p) = u;
  }
};
template <>
struct VIO<__nv_bfloat16, 4> {
  __device__ __forceinline__ static void ld(const __nv_bfloat16* p, float (&o)[4]) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.y));
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  }
  __device__ __forceinline__ static void st(__nv_bfloat16* p, const float (&v)[4]) {
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]);
    __nv_bfloat162 b = __floats2bfloat162_rn(v[2], v[3]);
    uint2 u;
    u.x = *reinterpret_cast<uint32_t*>(&a);
    u.y = *reinterpret_cast<uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p) = u;
  }
};

// N contiguous IO elements starting at p; 16-byte vectors when N * sizeof(T)
// is a multiple of 16 (callers guarantee the base is then 16-byte aligned).
template <class T, int N>
__device__ __forceinline__ void ld_contig(const T* p, T (&o)[N]) {
  if constexpr ((N * sizeof(T)) % 16 == 0) {
    constexpr int E = 16 / sizeof(T);
#pragma unroll
    for (int m = 0; m < N / E; ++m) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(p) + m);
      const T* t = reinterpret_cast<const T*>(&v);
#pragma unroll
      for (int e = 0; e < E; ++e) o[m * E + e] = t[e];
    }
  } else {
#pragma unroll
    for (int m = 0; m < N; ++m) o[m] = __ldg(p + m);
  }
}
template <class T, int N>
__device__ __forceinline__ void st_contig(T* p, const T (&v)[N]) {
  if constexpr ((N * sizeof(T)) % 16 == 0) {
    constexpr int E = 16 / sizeof(T);
#pragma unroll
    for (int m = 0; m < N / E; ++m) {
      float4 o;
      T* t = reinterpret_cast<T*>(&o);
#pragma unroll
      for (int e = 0; e < E; ++e) t[e] = v[m * E + e];
      reinterpret_cast<float4*>(p)[m] = o;
    }
  } else {
#pragma unroll
    for (int m = 0; m < N; ++m) p[m] = v[m];
  }
}

// ---------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------

enum FaceKind : int { kFaceNone = 0, kFacePressure = 1, kFaceVelocity = 2, kFaceZeroGrad = 3 };

struct FaceK {
  int kind;
  int axis;  // internal axis 0..2
  int side;  // 0 = min, 1 = max
  int ref_axis;
  double v[3];  // pressure: v[0] = rho_p; velocity: u in INTERNAL axis order
};

struct Geo {
  int n0, n1, n2;  // internal dims, a2 contiguous
  int nq;          // vectors per row (n2 / V)
  uint32_t nvec;   // n0 * n1 * nq
  int64_t ncell;   // n0 * n1 * n2 (stride between population planes)
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
  const void* pin;  // state in  (S)
  void* pout;       // state out (S)
  const void* f_in;   // AoS IO (prepare)
  void* f_out;        // AoS IO (final step)
  void* rho;
  void* vel;
  void* prs;
  uint32_t mflags;
};

constexpr uint32_t kMomDensityDev = 1u;

// Per-thread copy of the per-call parameters; device-resident values (traced
// scalars) override the host ones.
template <int Q, class R>
struct Params {
  R F[3];
  FaceK face[2];
};

template <int Q, class R>
__device__ __forceinline__ void load_params(const StepArgs& a, Params<Q, R>& p) {
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
#pragma unroll
  for (int d = 0; d < 3; ++d) p.F[d] = static_cast<R>(a.force[d]);
  p.face[0] = a.face[0];
  p.face[1] = a.face[1];
  if (a.dev_values != nullptr) {
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      const float* v = a.dev_values + 3 * f;
      if (p.face[f].kind == kFacePressure) {
        p.face[f].v[0] = v[0];
      } else if (p.face[f].kind == kFaceVelocity) {
        p.face[f].v[0] = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) p.face[f].v[d + sh] = v[d];
      }
    }
    if (a.force_mode == 1) {
      p.F[0] = 0;
#pragma unroll
      for (int d = 0; d < D; ++d) p.F[d + sh] = static_cast<R>(a.dev_values[6 + d]);
    }
  }
}

// ---------------------------------------------------------------------------
// Cell arithmetic (deviation form; all populations are offsets g = f - w)
// ---------------------------------------------------------------------------

template <int Q, class R>
struct Mom {
  R rd;    // rho - 1
  R rho;   // rho
  R u[3];  // velocity (internal axes), includes the Guo F/2 half step
};

// rho = sum f; rho u = sum f e + F/2; u = rho u / max(rho, 1e-10)  (lbm.py:209-239)
template <int Q, class R>
__device__ __forceinline__ Mom<Q, R> moments(const R (&f)[Q], const R (&F)[3]) {
  Mom<Q, R> m;
  R rd = 0, m0 = 0, m1 = 0, m2 = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    rd += f[q];
    if (Lat<Q>::c0(q) > 0) m0 += f[q];
    if (Lat<Q>::c0(q) < 0) m0 -= f[q];
    if (Lat<Q>::c1(q) > 0) m1 += f[q];
    if (Lat<Q>::c1(q) < 0) m1 -= f[q];
    if (Lat<Q>::c2(q) > 0) m2 += f[q];
    if (Lat<Q>::c2(q) < 0) m2 -= f[q];
  }
  const R half = R(0.5);
  m0 += half * F[0];
  m1 += half * F[1];
  m2 += half * F[2];
  m.rd = rd;
  m.rho = R(1) + rd;
  const R den = m.rho > R(1e-10) ? m.rho : R(1e-10);
  const R inv = R(1) / den;
  m.u[0] = m0 * inv;
  m.u[1] = m1 * inv;
  m.u[2] = m2 * inv;
  return m;
}

// BGK relax towards feq plus the Guo source term, in offsets:
//   geq_q = w_q (rho' + rho (3 eu + 4.5 eu^2 - 1.5 u^2))       (lbm.py:180-206)
//   S_q   = (1 - 1/(2 tau)) w_q (3 (e_q - u).F + 9 (e_q.u)(e_q.F))  (lbm.py:307-353)
//   p_q   = g_q - (g_q - geq_q) / tau + S_q                      (lbm.py:937-939)
template <int Q, class R>
__device__ __forceinline__ void collide(R (&f)[Q], const Mom<Q, R>& m, const R (&F)[3],
                                        R omega, R guo_c, bool has_force) {
  const R usq = m.u[0] * m.u[0] + m.u[1] * m.u[1] + m.u[2] * m.u[2];
  const R uF = m.u[0] * F[0] + m.u[1] * F[1] + m.u[2] * F[2];
  const R base = m.rd - m.rho * R(1.5) * usq;  // rho' + rho (-1.5 u^2)
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int a = Lat<Q>::c0(q), b = Lat<Q>::c1(q), c = Lat<Q>::c2(q);
    R eu = 0, eF = 0;
    if (a) { eu += a * m.u[0]; eF += a * F[0]; }
    if (b) { eu += b * m.u[1]; eF += b * F[1]; }
    if (c) { eu += c * m.u[2]; eF += c * F[2]; }
    const R w = static_cast<R>(Lat<Q>::w(q));
    const R geq = w * (base + m.rho * (R(3) * eu + R(4.5) * eu * eu));
    R p = f[q] + omega * (geq - f[q]);
    if (has_force) p += guo_c * w * (R(3) * (eF - uF) + R(9) * eu * eF);
    f[q] = p;
  }
}

// Reference Zou-He pressure face (lbm.py:425-510), in offsets.  Its closure
// u_n = +-(1 - (S_known + S_tang) / rho_p) carries no factor 2 on S_known;
// kept as is.  With W = sum of the known+tangential weights = 5/6 (both
// lattices), u_n = s (rho_p - 5/6 - G) / rho_p, G = sum of their offsets.
// Unknown q: f_q = f_opp + feq_q - feq_opp = f_opp + 6 w_q rho_p e_qa u_n.
template <int Q, class R>
__device__ __forceinline__ void face_pressure(R (&f)[Q], const FaceK& fc) {
  const int ax = fc.axis;
  const bool mn = fc.side == 0;
  R G = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (!unknown) G += f[q];
  }
  const double rho_p = fc.v[0];
  const R rho_c = static_cast<R>(rho_p > 1e-10 ? rho_p : 1e-10);
  const R c1 = static_cast<R>(rho_p - 5.0 / 6.0);
  R un = (c1 - G) / rho_c;
  if (!mn) un = -un;
  const R rp = static_cast<R>(rho_p);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (unknown) {
      const R w = static_cast<R>(Lat<Q>::w(q));
      f[q] = f[Lat<Q>::opp(q)] + R(6) * w * rp * static_cast<R>(cq) * un;
    }
  }
}

// Velocity face (extension): rho = (S_tang + 2 S_known) / (1 - s u_a), with
// W_tang + 2 W_known = 1 so rho = (1 + G_tang + 2 G_known) / (1 - s u_a);
// unknown q: f_q = f_opp + 6 w_q rho (e_q . u).
template <int Q, class R>
__device__ __forceinline__ void face_velocity(R (&f)[Q], const FaceK& fc) {
  const int ax = fc.axis;
  const bool mn = fc.side == 0;
  R G = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (cq == 0) G += f[q];
    else if (!unknown) G += R(2) * f[q];
  }
  const R u0 = static_cast<R>(fc.v[0]), u1 = static_cast<R>(fc.v[1]),
          u2 = static_cast<R>(fc.v[2]);
  const R ua = ax == 0 ? u0 : (ax == 1 ? u1 : u2);
  const R s = mn ? R(1) : R(-1);
  const R rho = (R(1) + G) / (R(1) - s * ua);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (unknown) {
      const R eu = Lat<Q>::c0(q) * u0 + Lat<Q>::c1(q) * u1 + Lat<Q>::c2(q) * u2;
      const R w = static_cast<R>(Lat<Q>::w(q));
      f[q] = f[Lat<Q>::opp(q)] + R(6) * w * rho * eu;
    }
  }
}

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Offset of population q that the reference's f_bc holds at cell (i0,i1,k):
// the pulled value p[x - e_q] or, in a wall cell, p[x + e_q] of opp(q).
template <int Q, class S>
__device__ __forceinline__ typename StoreT<S>::R fbc_at(const StepArgs& a, const S* pin, int q,
                                                        int i0, int i1, int k) {
  using R = typename StoreT<S>::R;
  const Geo& g = a.g;
  const bool wl = a.wall != nullptr &&
                  a.wall[(static_cast<int64_t>(i0) * g.n1 + i1) * g.n2 + k] != 0;
  const int s = wl ? 1 : -1;
  // resolve opp at runtime (q is runtime here)
  int c0 = 0, c1 = 0, c2 = 0, qs = q;
#pragma unroll
  for (int t = 0; t < Q; ++t) {
    if (t == q) {
      c0 = Lat<Q>::c0(t); c1 = Lat<Q>::c1(t); c2 = Lat<Q>::c2(t);
      qs = wl ? Lat<Q>::opp(t) : t;
    }
  }
  const int j0 = wrapi(i0 + s * c0, g.n0), j1 = wrapi(i1 + s * c1, g.n1), j2 = wrapi(k + s * c2, g.n2);
  R v = ld1<S>(pin + static_cast<int64_t>(qs) * g.ncell +
               (static_cast<int64_t>(j0) * g.n1 + j1) * g.n2 + j2);
  if constexpr (StoreT<S>::kScaled) {
    R w = 0;
#pragma unroll
    for (int t = 0; t < Q; ++t)
      if (t == qs) w = static_cast<R>(Lat<Q>::w(t));
    v *= w;
  }
  return v;
}

// Zero-gradient face (extension): unknown q <- f_bc at the neighbour one cell
// inwards (its post-stream, post-bounce value).
template <int Q, class S>
__device__ __forceinline__ void face_zero_gradient(typename StoreT<S>::R (&f)[Q], const StepArgs& a,
                                                   const S* pin, const FaceK& fc, int i0, int i1,
                                                   int k) {
  const int ax = fc.axis;
  const bool mn = fc.side == 0;
  const int d = mn ? 1 : -1;
  const int n0 = i0 + (ax == 0 ? d : 0), n1 = i1 + (ax == 1 ? d : 0), n2 = k + (ax == 2 ? d : 0);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int cq = comp<Q>(q, ax);
    const bool unknown = mn ? (cq > 0) : (cq < 0);
    if (unknown) f[q] = fbc_at<Q, S>(a, pin, q, n0, n1, n2);
  }
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Launch shape of the step kernels (threads per block, minimum resident
// blocks per SM for the register budget); overridable at compile time.
#ifndef LBM_STEP_BLOCK
#define LBM_STEP_BLOCK 128
#endif
#ifndef LBM_STEP_MINB
#define LBM_STEP_MINB 8
#endif
constexpr int kBlock = LBM_STEP_BLOCK;
constexpr int kMinBlocks = LBM_STEP_MINB;

enum StepMode : int { kOutState = 0, kOutAoS = 1 };

// Shared per-thread index decomposition.
struct Where {
  uint32_t gv;
  bool active;
  int i0, i1, k0;
  int jq;
  int64_t cell;  // linear index of the first of the V cells
};

template <int V>
__device__ __forceinline__ Where where_am_i(const Geo& g) {
  Where w;
  uint32_t gv = blockIdx.x * blockDim.x + threadIdx.x;
  w.active = gv < g.nvec;
  if (!w.active) gv = g.nvec - 1;  // keep every lane alive for the shuffles
  w.gv = gv;
  const uint32_t row = gv / static_cast<uint32_t>(g.nq);
  w.jq = static_cast<int>(gv - row * static_cast<uint32_t>(g.nq));
  w.i0 = static_cast<int>(row / static_cast<uint32_t>(g.n1));
  w.i1 = static_cast<int>(row - static_cast<uint32_t>(w.i0) * g.n1);
  w.k0 = w.jq * V;
  w.cell = static_cast<int64_t>(row) * g.n2 + w.k0;
  return w;
}

template <int Q, class IO, int V>
__device__ __forceinline__ void load_force(const StepArgs& a, int64_t cell, const IO* /*tag*/,
                                           typename StoreT<IO>::R (&Fv)[V][3]) {
  using R = typename StoreT<IO>::R;
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  IO buf[V * D];
  ld_contig<IO, V * D>(static_cast<const IO*>(a.force_field) + cell * D, buf);
#pragma unroll
  for (int r = 0; r < V; ++r) {
    Fv[r][0] = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) Fv[r][d + sh] = static_cast<R>(buf[r * D + d]);
  }
}

template <int Q, class IO, int V>
__device__ __forceinline__ void store_moments(const StepArgs& a, int64_t cell,
                                              const Mom<Q, typename StoreT<IO>::R> (&m)[V],
                                              const uint8_t (&wl)[V]) {
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  if (a.rho != nullptr) {
    IO d[V];
#pragma unroll
    for (int r = 0; r < V; ++r) d[r] = (a.mflags & kMomDensityDev) ? m[r].rd : m[r].rho;
    st_contig<IO, V>(static_cast<IO*>(a.rho) + cell, d);
  }
  if (a.prs != nullptr) {
    IO d[V];
#pragma unroll
    for (int r = 0; r < V; ++r) {
      if constexpr (sizeof(IO) == 8) d[r] = m[r].rho * (1.0 / 3.0);
      else d[r] = m[r].rho * static_cast<float>(1.0 / 3.0);
    }
    st_contig<IO, V>(static_cast<IO*>(a.prs) + cell, d);
  }
  if (a.vel != nullptr) {
    IO u[V * D];
#pragma unroll
    for (int r = 0; r < V; ++r)
#pragma unroll
      for (int d = 0; d < D; ++d) u[r * D + d] = wl[r] ? IO(0) : static_cast<IO>(m[r].u[d + sh]);
    st_contig<IO, V * D>(static_cast<IO*>(a.vel) + cell * D, u);
  }
}

template <int V>
__device__ __forceinline__ void load_wall(const StepArgs& a, int64_t cell, uint8_t (&wl)[V]) {
  if (a.wall == nullptr) {
#pragma unroll
    for (int r = 0; r < V; ++r) wl[r] = 0;
    return;
  }
  if constexpr (V == 4) {
    const uchar4 v = __ldg(reinterpret_cast<const uchar4*>(a.wall + cell));
    wl[0] = v.x; wl[1] = v.y; wl[2] = v.z; wl[3] = v.w;
  } else if constexpr (V == 2) {
    const uchar2 v = __ldg(reinterpret_cast<const uchar2*>(a.wall + cell));
    wl[0] = v.x; wl[1] = v.y;
  } else {
#pragma unroll
    for (int r = 0; r < V; ++r) wl[r] = __ldg(a.wall + cell + r);
  }
}

// Collide from a reference-layout state f (*grid_shape, Q): p = C(f).
// Cell-local; the first pass of every update / rollout.
template <int Q, class S, int V>
__global__ void __launch_bounds__(kBlock) k_prepare(const StepArgs a) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  const Geo& g = a.g;
  const Where w = where_am_i<V>(g);
  if (!w.active) return;
  Params<Q, R> prm;
  load_params<Q, R>(a, prm);

  IO raw[V * Q];
  ld_contig<IO, V * Q>(static_cast<const IO*>(a.f_in) + w.cell * Q, raw);
  R Fv[V][3];
  if (a.force_mode == 2) {
    load_force<Q, IO, V>(a, w.cell, static_cast<const IO*>(nullptr), Fv);
  } else {
#pragma unroll
    for (int r = 0; r < V; ++r)
#pragma unroll
      for (int d = 0; d < 3; ++d) Fv[r][d] = prm.F[d];
  }
  const bool has_force = a.force_mode != 0;
  const R omega = static_cast<R>(a.omega), guo_c = static_cast<R>(a.guo_c);
  R out[Q][V];
#pragma unroll
  for (int r = 0; r < V; ++r) {
    R f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if constexpr (sizeof(R) == 8) f[q] = raw[r * Q + q] - Lat<Q>::w(q);
      else f[q] = (raw[r * Q + q] - w_hi<Q>(q)) - w_lo<Q>(q);
    }
    const Mom<Q, R> m = moments<Q, R>(f, Fv[r]);
    collide<Q, R>(f, m, Fv[r], omega, guo_c, has_force);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      R v = f[q];
      if constexpr (StoreT<S>::kScaled) v *= static_cast<R>(1.0 / Lat<Q>::w(q));
      out[q][r] = v;
    }
  }
  S* po = static_cast<S*>(a.pout);
#pragma unroll
  for (int q = 0; q < Q; ++q) VIO<S, V>::st(po + static_cast<int64_t>(q) * g.ncell + w.cell, out[q]);
}

// One fused step: pull p -> wall swap -> faces (= reference f_bc) -> moments
// (reference outputs) -> collide (next p) or write f_bc (MODE kOutAoS).
template <int Q, class S, int V, int MODE>
__global__ void __launch_bounds__(kBlock, kMinBlocks) k_step(const StepArgs a) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  const Geo& g = a.g;
  const Where w = where_am_i<V>(g);
  const int lane = threadIdx.x & 31;
  const S* pin = static_cast<const S*>(a.pin);

  // Source rows of the pull x - e_q along a0 / a1 (periodic).
  const int i0m = w.i0 == 0 ? g.n0 - 1 : w.i0 - 1;
  const int i0p = w.i0 == g.n0 - 1 ? 0 : w.i0 + 1;
  const int i1m = w.i1 == 0 ? g.n1 - 1 : w.i1 - 1;
  const int i1p = w.i1 == g.n1 - 1 ? 0 : w.i1 + 1;

  R f[V][Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q), c2 = Lat<Q>::c2(q);
    const int s0 = c0 > 0 ? i0m : (c0 < 0 ? i0p : w.i0);
    const int s1 = c1 > 0 ? i1m : (c1 < 0 ? i1p : w.i1);
    const S* row = pin + static_cast<int64_t>(q) * g.ncell +
                   (static_cast<int64_t>(s0) * g.n1 + s1) * g.n2;
    if constexpr (V == 1) {
      const int ks = c2 > 0 ? (w.k0 == 0 ? g.n2 - 1 : w.k0 - 1)
                            : (c2 < 0 ? (w.k0 == g.n2 - 1 ? 0 : w.k0 + 1) : w.k0);
      f[0][q] = ld1<S>(row + ks);
    } else {
      R v[V];
      VIO<S, V>::ld(row + w.k0, v);
      if (c2 == 0) {
#pragma unroll
        for (int r = 0; r < V; ++r) f[r][q] = v[r];
      } else if (c2 > 0) {  // value at k - 1
        R left = __shfl_up_sync(0xffffffffu, v[V - 1], 1);
        if (lane == 0 || w.jq == 0) left = ld1<S>(row + (w.jq == 0 ? g.n2 - 1 : w.k0 - 1));
        f[0][q] = left;
#pragma unroll
        for (int r = 1; r < V; ++r) f[r][q] = v[r - 1];
      } else {  // value at k + 1
        R right = __shfl_down_sync(0xffffffffu, v[0], 1);
        if (lane == 31 || w.jq == g.nq - 1) right = ld1<S>(row + (w.jq == g.nq - 1 ? 0 : w.k0 + V));
#pragma unroll
        for (int r = 0; r < V - 1; ++r) f[r][q] = v[r + 1];
        f[V - 1][q] = right;
      }
    }
    if constexpr (StoreT<S>::kScaled) {
      const R ws = static_cast<R>(Lat<Q>::w(q));
#pragma unroll
      for (int r = 0; r < V; ++r) f[r][q] *= ws;
    }
  }
  if (!w.active) return;  // past the shuffles: tail lanes may leave

  Params<Q, R> prm;
  load_params<Q, R>(a, prm);
  uint8_t wl[V];
  load_wall<V>(a, w.cell, wl);

  R Fv[V][3];
  if (a.force_mode == 2) {
    load_force<Q, IO, V>(a, w.cell, static_cast<const IO*>(nullptr), Fv);
  } else {
#pragma unroll
    for (int r = 0; r < V; ++r)
#pragma unroll
      for (int d = 0; d < 3; ++d) Fv[r][d] = prm.F[d];
  }

  Mom<Q, R> m[V];
#pragma unroll
  for (int r = 0; r < V; ++r) {
    // Wall-node swap (lbm.py:944-948): a wall cell takes f_str[..., opp].
    if (wl[r]) {
#pragma unroll
      for (int q = 1; q < Q; ++q) {
        if (q < Lat<Q>::opp(q)) {
          const R t = f[r][q];
          f[r][q] = f[r][Lat<Q>::opp(q)];
          f[r][Lat<Q>::opp(q)] = t;
        }
      }
    }
    // Faces: inlet first, then outlet (lbm.py:950-968); wall face cells untouched.
    const int k = w.k0 + r;
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
      const FaceK& fc = prm.face[fi];
      if (fc.kind == kFaceNone || wl[r]) continue;
      const int coord = fc.axis == 0 ? w.i0 : (fc.axis == 1 ? w.i1 : k);
      const int nax = fc.axis == 0 ? g.n0 : (fc.axis == 1 ? g.n1 : g.n2);
      if (coord != (fc.side == 0 ? 0 : nax - 1)) continue;
      if (fc.kind == kFacePressure) face_pressure<Q, R>(f[r], fc);
      else if (fc.kind == kFaceVelocity) face_velocity<Q, R>(f[r], fc);
      else face_zero_gradient<Q, S>(f[r], a, pin, fc, w.i0, w.i1, k);
    }
    m[r] = moments<Q, R>(f[r], Fv[r]);
  }
  store_moments<Q, IO, V>(a, w.cell, m, wl);

  if constexpr (MODE == kOutAoS) {
    // Reference state f (*grid_shape, Q) = w + offset.
    IO raw[V * Q];
#pragma unroll
    for (int r = 0; r < V; ++r)
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        if constexpr (sizeof(R) == 8) raw[r * Q + q] = Lat<Q>::w(q) + f[r][q];
        else raw[r * Q + q] = w_hi<Q>(q) + (f[r][q] + w_lo<Q>(q));
      }
    st_contig<IO, V * Q>(static_cast<IO*>(a.f_out) + w.cell * Q, raw);
  } else {
    const bool has_force = a.force_mode != 0;
    const R omega = static_cast<R>(a.omega), guo_c = static_cast<R>(a.guo_c);
    R out[Q][V];
#pragma unroll
    for (int r = 0; r < V; ++r) {
      collide<Q, R>(f[r], m[r], Fv[r], omega, guo_c, has_force);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        R v = f[r][q];
        if constexpr (StoreT<S>::kScaled) v *= static_cast<R>(1.0 / Lat<Q>::w(q));
        out[q][r] = v;
      }
    }
    S* po = static_cast<S*>(a.pout);
#pragma unroll
    for (int q = 0; q < Q; ++q) VIO<S, V>::st(po + static_cast<int64_t>(q) * g.ncell + w.cell, out[q]);
  }
}

// f = feq(rho, u) in the reference layout (lbm.py:180-206, 719-745).
template <int Q, class IO>
__global__ void __launch_bounds__(kBlock) k_equilibrium(Geo g, const IO* rho, const IO* u, IO* f) {
  using R = typename StoreT<IO>::R;
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  const int64_t cell = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (cell >= g.ncell) return;
  Mom<Q, R> m;
  m.rho = rho ? static_cast<R>(rho[cell]) : R(1);
  m.rd = m.rho - R(1);
  m.u[0] = m.u[1] = m.u[2] = 0;
  if (u)
    for (int d = 0; d < D; ++d) m.u[d + sh] = static_cast<R>(u[cell * D + d]);
  R gq[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) gq[q] = 0;
  const R F[3] = {0, 0, 0};
  // omega = 1: p = geq exactly
  collide<Q, R>(gq, m, F, R(1), R(0), false);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if constexpr (sizeof(R) == 8) f[cell * Q + q] = Lat<Q>::w(q) + gq[q];
    else f[cell * Q + q] = w_hi<Q>(q) + (gq[q] + w_lo<Q>(q));
  }
}

// FP64 mass / momentum partial sums: block b writes part[4 b .. 4 b + 3].
template <int Q, class IO>
__global__ void __launch_bounds__(kBlock) k_mass_momentum_part(Geo g, const IO* f, double* part) {
  double acc[4] = {0, 0, 0, 0};
  for (int64_t cell = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; cell < g.ncell;
       cell += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double v = static_cast<double>(f[cell * Q + q]) - Lat<Q>::w(q);
      acc[0] += v;
      acc[1] += Lat<Q>::c0(q) * v;
      acc[2] += Lat<Q>::c1(q) * v;
      acc[3] += Lat<Q>::c2(q) * v;
    }
  }
  __shared__ double red[kBlock / 32][4];
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
    for (int wi = 0; wi < kBlock / 32; ++wi) v += red[wi][threadIdx.x];
    part[4 * blockIdx.x + threadIdx.x] = v;
  }
}

// Final fixed-order reduction of nparts partials; out = {mass, momentum (ref order)}.
template <int Q>
__global__ void __launch_bounds__(kBlock) k_mass_momentum_final(const double* part, int nparts,
                                                                double ncell, double* out) {
  __shared__ double red[kBlock / 32][4];
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
    for (int wi = 0; wi < kBlock / 32; ++wi)
      for (int c = 0; c < 4; ++c) s[c] += red[wi][c];
    constexpr int D = Lat<Q>::D;
    out[0] = ncell + s[0];
    // internal axes -> reference order
    for (int d = 0; d < D; ++d) out[1 + d] = s[1 + d + (3 - D)];
    for (int d = D; d < 3; ++d) out[1 + d] = 0.0;
  }
}

}  // namespace lbm
