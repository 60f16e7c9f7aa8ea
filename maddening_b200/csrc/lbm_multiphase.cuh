// Shan-Chen multiphase step of the pipe node (MADDENING LBMPipeNode.update
// with G != 0, src/maddening/nodes/lbm_pipe.py:751-864; the interaction force
// is _shan_chen_force, lbm_pipe.py:321-375):
//   rho, u   = moments(f) (no half-force step), u = m / max(rho, 1e-10)
//   psi(y)   = psi_wall in walls, else rho_0 (1 - exp(-rho(y) / rho_0))
//   F        = propeller + gravity + (0 in walls) -G psi(x) sum_q w_q psi(x + e_q) e_q
//   u_s      = u + F / max(rho, 0.01), scaled down to |u_s| <= 0.25
//   f*       = f - (f - feq(rho, u)) / tau + (feq(rho, u_s) - feq(rho, u))   (exact difference)
//   f_bc     = periodic stream of f*, wall-node swap
//   floor    : where sum f_bc < 0.01, f_bc *= 0.01 / sum f_bc and rho = 0.01
//   outputs  : rho, u = moments(f_bc) (0 in walls), tracer = clip((rho - rho_gas) /
//              (rho_liquid - rho_gas), 0, 1) (0 in walls); tracer_f passes through.
//
// The force at x needs psi at the 18 neighbours, i.e. the density of every
// cell before any cell collides, so a step is two passes over planes that
// hold the POST-collision populations p (FP32, FP64 for FP64 plans), one per
// direction, both pulling f_str(x)_q = p_q(x - e_q) as the single-phase step
// does:
//   k_mp_density  pulls, sums, applies the density floor, writes psi (one
//                 plane);
//   k_mp_collide  pulls again, applies the same floor, swaps wall cells,
//                 collides with psi of the neighbours and stores p(x) in
//                 place: every warp store is one aligned 128-byte run.
// The first step collides the reference f (read through shared memory in
// its (grid, 19) layout); the last pass pulls the state into the reference
// f_bc and the outputs.  Every sum runs in the order of the push form this
// replaced (f_str before the wall swap), so the outputs are bit-identical.
// Traffic per cell and step: 19 loads + 1 psi store, then 19 loads + 19
// stores + the psi loads (mostly cache hits).
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

struct MPArgs {
  StepArgs s;            // geometry, wall, omega, pipe force (force_mode 3 fields)
  double G, rho0;        // interaction strength, pseudopotential density
  double psi_wall;       // rho_0 (1 - exp(-rho_wall / rho_0))
  double rho_gas, drho;  // tracer = (rho - rho_gas) / drho, drho = rho_liquid - rho_gas
  const void* fin;       // population planes
  void* fout;
  void* psi;             // psi plane
  const void* f_aos_in;  // (grid, 19) reference layout (first pass)
  void* f_aos_out;       // (grid, 19) reference layout (last pass)
  void* rho_out;         // grid (last pass)
  void* vel_out;         // (grid, 3) (last pass)
  void* tracer_out;      // grid (last pass; NULL = not written)
};

constexpr int kMPFirst = 0;  // f from the reference layout, no floor, psi
constexpr int kMPStep = 1;   // floor in place, psi
constexpr int kMPLast = 2;   // floor, f to the reference layout, outputs

template <class R>
__device__ __forceinline__ R sum19(const R (&f)[19]) {
  R s = f[0];
#pragma unroll
  for (int q = 1; q < 19; ++q) s = add_r(s, f[q]);
  return s;
}

template <class R>
__device__ __forceinline__ void mom19(const R (&f)[19], R (&m)[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    R acc = 0;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
      const int e = d == 0 ? Lat<19>::c0(q) : (d == 1 ? Lat<19>::c1(q) : Lat<19>::c2(q));
      if (e > 0) acc = add_r(acc, f[q]);
      if (e < 0) acc = sub_r(acc, f[q]);
    }
    m[d] = acc;
  }
}

// Exchange slots q and opp(q): the wall-node swap of a wall cell.
template <class R>
__device__ __forceinline__ void swap_opp(R (&f)[19]) {
#pragma unroll
  for (int q = 1; q < 19; ++q) {
    const int o = Lat<19>::opp(q);
    if (q < o) {
      const R t = f[q];
      f[q] = f[o];
      f[o] = t;
    }
  }
}

__device__ __forceinline__ float sqrt_r(float x) { return __fsqrt_rn(x); }
__device__ __forceinline__ double sqrt_r(double x) { return __dsqrt_rn(x); }
__device__ __forceinline__ float expm1_r(float x) { return expm1f(x); }
__device__ __forceinline__ double expm1_r(double x) { return expm1(x); }

// psi(rho) = rho_0 (1 - exp(-rho / rho_0)), lbm_pipe.py:301-318, written with
// expm1 so that small densities keep their relative precision.
template <class R>
__device__ __forceinline__ R psi_of(R rho, R rho0) {
  return mul_r(rho0, -expm1_r(div_r(-rho, rho0)));
}

// Offsets of the periodic neighbours x -/+ 1 along each axis.
struct MPNbr {
  int32_t o0m, o0p, o1m, o1p, o2m, o2p;
};

__device__ __forceinline__ MPNbr mp_nbr(const Geo& g, const Cell& x) {
  const int32_t pl = static_cast<int32_t>(g.plane), rw = static_cast<int32_t>(g.n2);
  MPNbr o;
  o.o0m = x.i0 == 0 ? (static_cast<int32_t>(g.n0) - 1) * pl : -pl;
  o.o0p = x.i0 + 1 == g.n0 ? -(static_cast<int32_t>(g.n0) - 1) * pl : pl;
  o.o1m = x.i1 == 0 ? (static_cast<int32_t>(g.n1) - 1) * rw : -rw;
  o.o1p = x.i1 + 1 == g.n1 ? -(static_cast<int32_t>(g.n1) - 1) * rw : rw;
  o.o2m = x.k == 0 ? rw - 1 : -1;
  o.o2p = x.k + 1 == g.n2 ? 1 - rw : 1;
  return o;
}

// The cell x + s e_q (s = +1 or -1), periodic.
__device__ __forceinline__ uint32_t mp_at(const MPNbr& o, uint32_t c, int q, int s) {
  const int e0 = s * Lat<19>::c0(q), e1 = s * Lat<19>::c1(q), e2 = s * Lat<19>::c2(q);
  int32_t d = 0;
  if (e0) d += e0 > 0 ? o.o0p : o.o0m;
  if (e1) d += e1 > 0 ? o.o1p : o.o1m;
  if (e2) d += e2 > 0 ? o.o2p : o.o2m;
  return static_cast<uint32_t>(static_cast<int32_t>(c) + d);
}

// f_str of cell c: population q pulled from x - e_q of the post-collision planes.
template <class R>
__device__ __forceinline__ void mp_pull(const MPArgs& a, const MPNbr& o, uint32_t c, R (&f)[19]) {
  const R* fi = static_cast<const R*>(a.fin);
  const uint32_t n = a.s.g.ncell;
#pragma unroll
  for (int q = 0; q < 19; ++q) f[q] = __ldg(fi + static_cast<size_t>(q) * n + mp_at(o, c, q, -1));
}

// The floor of lbm_pipe.py:838-848 on the pulled populations f (sum s0):
// scaled by 0.01 / s0 when s0 < 0.01; returns the sum the step continues with.
template <class R>
__device__ __forceinline__ R mp_floor(R (&f)[19], R s0) {
  const R floor = static_cast<R>(0.01);
  if (!(s0 < floor)) return s0;
  const R ratio = div_r(floor, s0 > R(1e-20) ? s0 : R(1e-20));
#pragma unroll
  for (int q = 0; q < 19; ++q) f[q] = mul_r(f[q], ratio);
  return sum19(f);
}

// Density pass of cell c.  kMPFirst: f is the reference f_bc (row of the
// staged tile), psi without a floor; kMPStep: f pulled, floor, psi;
// kMPLast: f pulled, floor, the reference f_bc and the outputs.
template <class R, int MODE>
__device__ __forceinline__ void density_cell(const MPArgs& a, uint32_t c, R (&f)[19]) {
  const bool wall = a.s.wall != nullptr && a.s.wall[c] != 0;
  const R s0 = sum19(f);  // the new density before the floor (f_str order)
  R m[3] = {0, 0, 0};
  if (MODE == kMPLast) {
    if (wall) swap_opp(f);  // to f_bc (no velocity is taken in walls)
    else mom19(f, m);       // the output velocity is taken before the floor
  }
  R s = s0, rho_out = s0;
  if (MODE != kMPFirst && s0 < static_cast<R>(0.01)) {
    s = mp_floor(f, s0);
    rho_out = static_cast<R>(0.01);
  }
  if constexpr (MODE != kMPLast) {
    static_cast<R*>(a.psi)[c] =
        wall ? static_cast<R>(a.psi_wall) : psi_of(s, static_cast<R>(a.rho0));
    return;
  }
  R* out_row = aos_tile<19, R>() + threadIdx.x * 19;
#pragma unroll
  for (int q = 0; q < 19; ++q) out_row[q] = f[q];
  if (a.rho_out != nullptr) static_cast<R*>(a.rho_out)[c] = rho_out;
  if (a.vel_out != nullptr) {
    const R den = s0 > R(1e-10) ? s0 : R(1e-10);
    R* v = static_cast<R*>(a.vel_out) + static_cast<size_t>(c) * 3;
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = wall ? R(0) : div_r(m[d], den);
  }
  if (a.tracer_out != nullptr) {
    R t = div_r(sub_r(rho_out, static_cast<R>(a.rho_gas)), static_cast<R>(a.drho));
    t = t < R(0) ? R(0) : (t > R(1) ? R(1) : t);
    static_cast<R*>(a.tracer_out)[c] = wall ? R(0) : t;
  }
}

template <class R, int MODE>
__global__ void __launch_bounds__(kBlock) k_mp_density(const MPArgs a) {
  const Geo& g = a.s.g;
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  R f[19];
  // the first and last passes stage the reference layout: every thread of
  // the block reaches the tile's barriers
  if constexpr (MODE == kMPFirst) {
    const R* row = aos_fill<19, R>(static_cast<const R*>(a.f_aos_in), blockIdx.x * kBlock, g.ncell);
    if (c < g.ncell) {
#pragma unroll
      for (int q = 0; q < 19; ++q) f[q] = row[q];
      density_cell<R, MODE>(a, c, f);  // (a wall cell's psi is psi_wall: no order issue)
    }
  } else {
    if (c < g.ncell) {
      const Cell x = locate(g, c);
      mp_pull<R>(a, mp_nbr(g, x), c, f);
      density_cell<R, MODE>(a, c, f);
    }
    if constexpr (MODE == kMPLast)
      aos_flush<19, R>(static_cast<R*>(a.f_aos_out), blockIdx.x * kBlock, g.ncell);
  }
}

// Collide with the Shan-Chen force and exact-difference forcing; the cell's
// own p is stored in place.  FIRST: the populations come from the reference
// f_bc (staged tile), no floor.
template <class R, bool FIRST>
__global__ void __launch_bounds__(kBlock) k_mp_collide(const MPArgs a) {
  const Geo& g = a.s.g;
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  R f[19];
  const R* row = nullptr;
  if constexpr (FIRST)
    row = aos_fill<19, R>(static_cast<const R*>(a.f_aos_in), blockIdx.x * kBlock, g.ncell);
  if (c >= g.ncell) return;
  const Cell x = locate(g, c);
  const MPNbr o = mp_nbr(g, x);
  // psi of the cell and of its 18 neighbours, loaded ahead of the wall test so
  // that they travel with the population loads (only fluid cells use them)
  const R* psi = static_cast<const R*>(a.psi);
  R pn[19];
  pn[0] = __ldg(psi + c);
#pragma unroll
  for (int q = 1; q < 19; ++q) pn[q] = __ldg(psi + mp_at(o, c, q, 1));
  const uint8_t* wm = a.s.wall;
  const bool wall = wm != nullptr && wm[c] != 0;
  R rho;
  if constexpr (FIRST) {
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = row[q];
    if (wall) swap_opp(f);  // the f_str order of the sum
    rho = sum19(f);
  } else {
    mp_pull<R>(a, o, c, f);
    rho = mp_floor(f, sum19(f));
  }
  if (wall) swap_opp(f);  // the wall-node swap: f_bc
  R m[3];
  mom19(f, m);
  const R inv_den = rcp_r(rho > R(1e-10) ? rho : R(1e-10));
  R u[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) u[d] = mul_r(m[d], inv_den);
  R F[3];
  pipe_force<R>(a.s, c, wall, F);
  if (!wall) {
    // sum_q w_q psi(x + e_q) e_q = (2 S_axis + S_diag) / 36
    R s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0};
#pragma unroll
    for (int q = 1; q < 19; ++q) {
      const int e0 = Lat<19>::c0(q), e1 = Lat<19>::c1(q), e2 = Lat<19>::c2(q);
      const R p = pn[q];
      R(&acc)[3] = q <= 6 ? s1 : s2;
      if (e0) acc[0] = e0 > 0 ? add_r(acc[0], p) : sub_r(acc[0], p);
      if (e1) acc[1] = e1 > 0 ? add_r(acc[1], p) : sub_r(acc[1], p);
      if (e2) acc[2] = e2 > 0 ? add_r(acc[2], p) : sub_r(acc[2], p);
    }
    const R coef = mul_r(static_cast<R>(-a.G), pn[0]);
    const R inv36 = static_cast<R>(1.0 / 36.0);
#pragma unroll
    for (int d = 0; d < 3; ++d) F[d] = fma_r(coef, mul_r(fma_r(R(2), s1[d], s2[d]), inv36), F[d]);
  }
  // shifted velocity u + F / max(rho, 0.01), clamped to |u_s| <= 0.25
  const R inv_rs = rcp_r(rho > R(0.01) ? rho : static_cast<R>(0.01));
  R us[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) us[d] = fma_r(F[d], inv_rs, u[d]);
  const R umag = sqrt_r(fma_r(us[0], us[0], fma_r(us[1], us[1], mul_r(us[2], us[2]))));
  if (umag > R(0.25)) {
    const R scale = mul_r(R(0.25), rcp_r(umag));
#pragma unroll
    for (int d = 0; d < 3; ++d) us[d] = mul_r(us[d], scale);
  }
  const R omega = static_cast<R>(a.s.omega);
  const R usq_b = fma_r(u[0], u[0], fma_r(u[1], u[1], mul_r(u[2], u[2])));
  const R usq_s = fma_r(us[0], us[0], fma_r(us[1], us[1], mul_r(us[2], us[2])));
  const R dusq = sub_r(usq_s, usq_b);
  const R r36 = mul_r(rho, static_cast<R>(1.0 / 36.0));
  R* fo = static_cast<R*>(a.fout);
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const R wr = mul_r(static_cast<R>(Lat<19>::wr(q)), r36);  // w_q rho
    const R eb = dot_e(Lat<19>::c0(q), Lat<19>::c1(q), Lat<19>::c2(q), u);
    const R es = dot_e(Lat<19>::c0(q), Lat<19>::c1(q), Lat<19>::c2(q), us);
    // feq(rho, u) = w rho (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u.u)
    const R feq = mul_r(wr, fma_r(eb, fma_r(R(4.5), eb, R(3)), fma_r(R(-1.5), usq_b, R(1))));
    // feq(rho, u_s) - feq(rho, u) = w rho (3 de + 4.5 de (es + eb) - 1.5 d(u.u))
    const R de = sub_r(es, eb);
    const R dfeq =
        mul_r(wr, fma_r(de, fma_r(R(4.5), add_r(es, eb), R(3)), mul_r(R(-1.5), dusq)));
    fo[static_cast<size_t>(q) * g.ncell + c] = add_r(fma_r(-omega, sub_r(f[q], feq), f[q]), dfeq);
  }
}

}  // namespace lbm
