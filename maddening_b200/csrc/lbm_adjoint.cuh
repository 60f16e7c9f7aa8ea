// Adjoint (reverse-mode) kernels of the lattice-Boltzmann rollout.
//
// Forward, per step n (the reference's LBMNode.update, lbm.py:899-986, without faces):
//   f^n = B S p^{n-1}   (pull-stream S, wall-node swap B; cell-local B)
//   (rho^n, u^n) = M(f^n; F)   with u = (sum f e + F/2) / rho
//   p^n = C(f^n) = f^n - omega (f^n - feq(rho^n, u^n)) + S_guo(u^n, F)
// Reverse, with lambda^n = dL/df^n and mu^n = B^T lambda^n (the wall swap is its
// own transpose):
//   nu_q(x)      = mu^{n+1}(x + e_q)_q          (S^T: a pull with the opposite shift)
//   lambda^n_r   = (1 - omega) nu_r + h + G . e_r
//   dL/dF(x)    += G / 2 + c b
// where, with P_q(u) = 1 + 3 e_q.u + 4.5 (e_q.u)^2 - 1.5 u^2 and its gradient
// grad P_q = 3 e_q + 9 (e_q.u) e_q - 3 u,
//   a = sum_q w_q nu_q P_q,  b = sum_q w_q nu_q grad P_q,
//   d = c sum_q w_q nu_q (-3 F + 9 (e_q.F) e_q),  c = 1 - 1/(2 tau),
//   G = omega b + d / rho,  h = omega a - G . u.
// (From dfeq_q/df_r = w_q [P_q + grad P_q . (e_r - u)], du/df_r = (e_r - u)/rho,
// du/dF = I/(2 rho); the Guo term depends on f only through u.)
// The Jacobian needs only (rho^n, u^n, F): the recomputed forward stores them
// (16 B per cell and step) instead of the populations.
// Adjoint populations are kept in f units (dL/df), one plane per direction.
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

struct AdjArgs {
  Geo g;
  double omega, guo_c;
  int force_mode;
  double force[3];  // internal axis order
  const void* force_field;
  const uint8_t* wall;
  const void* min;  // mu^{n+1} (S), direction q of cell c at [q * ncell + c]
  void* mout;       // mu^n (S)
  const void* rho;         // rho^n  (IO, grid)
  const void* vel;         // u^n    (IO, (grid, D), not zeroed in walls)
  double* dF;              // dL/dF accumulator ((grid, D), reference order) or null
  void* grad_f0;           // (grid, Q) IO output of the last reverse step, or null
  const void* g_rho;       // dL/d density^T  (IO, grid) or null
  const void* g_vel;       // dL/d velocity^T (IO, (grid, D)) or null
  const void* g_f;         // dL/d f^T        (IO, (grid, Q)) or null
};

enum AdjMode : int { kAdjOutState = 0, kAdjOutAoS = 1 };

template <int Q, class S>
__device__ __forceinline__ void adj_store(const AdjArgs& a, uint32_t c,
                                          typename StoreT<S>::R (&lam)[Q], bool wall) {
  if (wall) {
#pragma unroll
    for (int q = 1; q < Q; ++q) {
      if (q < Lat<Q>::opp(q)) {
        const auto t = lam[q];
        lam[q] = lam[Lat<Q>::opp(q)];
        lam[Lat<Q>::opp(q)] = t;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < Q; ++q)
    static_cast<S*>(a.mout)[static_cast<uint32_t>(q) * a.g.ncell + c] = from_r<S>(lam[q]);
}

// lambda^T from the gradients of the step-T outputs (density, velocity with
// u = 0 in walls, and f itself); dF starts at the direct term du/dF = 1/(2 rho).
template <int Q, class S>
__global__ void __launch_bounds__(kBlock) k_adj_init(const AdjArgs a) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  if (c >= a.g.ncell) return;
  const bool wall = a.wall != nullptr && a.wall[c] != 0;
  const R rho = static_cast<R>(static_cast<const IO*>(a.rho)[c]);
  R u[3] = {0, 0, 0}, gu[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) u[d + sh] = static_cast<R>(static_cast<const IO*>(a.vel)[c * D + d]);
  const R grho = a.g_rho ? static_cast<R>(static_cast<const IO*>(a.g_rho)[c]) : R(0);
  if (a.g_vel && !wall) {
#pragma unroll
    for (int d = 0; d < D; ++d)
      gu[d + sh] = static_cast<R>(static_cast<const IO*>(a.g_vel)[c * D + d]);
  }
  const R inv = R(1) / rho;
  const R gu_u = (gu[0] * u[0] + gu[1] * u[1] + gu[2] * u[2]) * inv;
  R lam[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    R v = grho - gu_u;
    if (Lat<Q>::c0(q)) v += Lat<Q>::c0(q) > 0 ? gu[0] * inv : -gu[0] * inv;
    if (Lat<Q>::c1(q)) v += Lat<Q>::c1(q) > 0 ? gu[1] * inv : -gu[1] * inv;
    if (Lat<Q>::c2(q)) v += Lat<Q>::c2(q) > 0 ? gu[2] * inv : -gu[2] * inv;
    if (a.g_f) v += static_cast<R>(static_cast<const IO*>(a.g_f)[static_cast<size_t>(c) * Q + q]);
    lam[q] = v;
  }
  if (a.dF != nullptr) {
#pragma unroll
    for (int d = 0; d < D; ++d) a.dF[static_cast<size_t>(c) * D + d] = 0.5 * gu[d + sh] * inv;
  }
  adj_store<Q, S>(a, c, lam, wall);
}

// One reverse step (see the header comment).  MODE kAdjOutAoS writes lambda^0
// = dL/df^0 in the reference (grid, Q) layout instead of mu.
template <int Q, class S, bool FORCE, int MODE>
__global__ void __launch_bounds__(kBlock, min_blocks<S>()) k_adj_step(const AdjArgs a) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  constexpr int D = Lat<Q>::D;
  constexpr int sh = 3 - D;
  const Geo& g = a.g;
  const uint32_t cidx = blockIdx.x * kBlock + threadIdx.x;
  if (cidx >= g.ncell) return;
  const Cell x = locate(g, cidx);

  // nu_q = mu(x + e_q)_q: source rows at +e_q (periodic).
  const uint32_t dm0 = x.i0 == 0 ? (g.n0 - 1) * g.plane : 0u - g.plane;
  const uint32_t dp0 = x.i0 == g.n0 - 1 ? 0u - (g.n0 - 1) * g.plane : g.plane;
  const uint32_t dm1 = x.i1 == 0 ? (g.n1 - 1) * g.n2 : 0u - g.n2;
  const uint32_t dp1 = x.i1 == g.n1 - 1 ? 0u - (g.n1 - 1) * g.n2 : g.n2;
  const uint32_t km = x.k == 0 ? g.n2 - 1 : x.k - 1;
  const uint32_t kp = x.k == g.n2 - 1 ? 0 : x.k + 1;
  R nu[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q), c2 = Lat<Q>::c2(q);
    uint32_t off = x.row;
    if (c0 > 0) off += dp0;
    if (c0 < 0) off += dm0;
    if (c1 > 0) off += dp1;
    if (c1 < 0) off += dm1;
    off += c2 > 0 ? kp : (c2 < 0 ? km : x.k);
    nu[q] = ld_pop<S>(static_cast<const S*>(a.min) + (static_cast<uint32_t>(q) * g.ncell + off));
  }

  const bool wall = a.wall != nullptr && __ldg(a.wall + cidx) != 0;
  const R rho = static_cast<R>(static_cast<const IO*>(a.rho)[cidx]);
  R u[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d)
    u[d + sh] = static_cast<R>(static_cast<const IO*>(a.vel)[static_cast<size_t>(cidx) * D + d]);
  R F[3] = {0, 0, 0};
  if (FORCE) {
    if (a.force_mode == 2) load_force<Q, IO>(a.force_field, cidx, F);
    else {
#pragma unroll
      for (int d = 0; d < 3; ++d) F[d] = static_cast<R>(a.force[d]);
    }
  }
  const R omega = static_cast<R>(a.omega), cg = static_cast<R>(a.guo_c);
  const R usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];

  // Pair sums: sigma = nu_q + nu_opp, tau = nu_q - nu_opp.
  R sw = static_cast<R>(Lat<Q>::w(0)) * nu[0];  // sum_q w_q nu_q
  R aa = 0;                                     // sum_pairs w (4.5 sigma eu^2 + 3 tau eu)
  R bb[3] = {0, 0, 0};                          // sum_pairs w (3 tau + 9 sigma eu) e_q
  R dd[3] = {0, 0, 0};                          // sum_pairs w sigma eF e_q
#pragma unroll
  for (int q = 1; q < Q; ++q) {
    if (q > Lat<Q>::opp(q)) continue;
    const int o = Lat<Q>::opp(q);
    const int e0 = Lat<Q>::c0(q), e1 = Lat<Q>::c1(q), e2 = Lat<Q>::c2(q);
    const R w = static_cast<R>(Lat<Q>::w(q));
    const R sg = nu[q] + nu[o], tu = nu[q] - nu[o];
    R eu = 0;
    if (e0) eu += e0 > 0 ? u[0] : -u[0];
    if (e1) eu += e1 > 0 ? u[1] : -u[1];
    if (e2) eu += e2 > 0 ? u[2] : -u[2];
    sw += w * sg;
    aa += w * (R(4.5) * sg * eu * eu + R(3) * tu * eu);
    const R cb = w * (R(3) * tu + R(9) * sg * eu);
    if (e0) bb[0] += e0 > 0 ? cb : -cb;
    if (e1) bb[1] += e1 > 0 ? cb : -cb;
    if (e2) bb[2] += e2 > 0 ? cb : -cb;
    if (FORCE) {
      R eF = 0;
      if (e0) eF += e0 > 0 ? F[0] : -F[0];
      if (e1) eF += e1 > 0 ? F[1] : -F[1];
      if (e2) eF += e2 > 0 ? F[2] : -F[2];
      const R cd = w * sg * eF;
      if (e0) dd[0] += e0 > 0 ? cd : -cd;
      if (e1) dd[1] += e1 > 0 ? cd : -cd;
      if (e2) dd[2] += e2 > 0 ? cd : -cd;
    }
  }
  const R A = sw * (R(1) - R(1.5) * usq) + aa;
  R b[3], G[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    b[d] = bb[d] - R(3) * u[d] * sw;
    R dv = 0;
    if (FORCE) dv = cg * (R(9) * dd[d] - R(3) * F[d] * sw);
    G[d] = omega * b[d] + dv / rho;
  }
  const R h = omega * A - (G[0] * u[0] + G[1] * u[1] + G[2] * u[2]);
  const R keep = R(1) - omega;
  R lam[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    R v = keep * nu[q] + h;
    if (Lat<Q>::c0(q)) v += Lat<Q>::c0(q) > 0 ? G[0] : -G[0];
    if (Lat<Q>::c1(q)) v += Lat<Q>::c1(q) > 0 ? G[1] : -G[1];
    if (Lat<Q>::c2(q)) v += Lat<Q>::c2(q) > 0 ? G[2] : -G[2];
    lam[q] = v;
  }
  if (a.dF != nullptr) {
    double* p = a.dF + static_cast<size_t>(cidx) * D;
#pragma unroll
    for (int d = 0; d < D; ++d)
      p[d] += static_cast<double>(R(0.5) * G[d + sh] + cg * b[d + sh]);
  }
  if constexpr (MODE == kAdjOutAoS) {
    IO* o = static_cast<IO*>(a.grad_f0) + static_cast<size_t>(cidx) * Q;
#pragma unroll
    for (int q = 0; q < Q; ++q) o[q] = static_cast<IO>(lam[q]);
  } else {
    adj_store<Q, S>(a, cidx, lam, wall);
  }
}

// Sum of a (grid, D) FP64 field into out[0..D-1] (fixed order, two passes via
// the mass/momentum partial kernels' layout: block b writes part[4 b + d]).
template <int D>
__global__ void __launch_bounds__(kReduceThreads) k_field_sum_part(const double* field,
                                                                   uint32_t ncell, double* part) {
  double acc[3] = {0, 0, 0};
  for (size_t c = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; c < ncell;
       c += static_cast<size_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int d = 0; d < D; ++d) acc[d] += field[c * D + d];
  }
  __shared__ double red[kReduceThreads / 32][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double v = acc[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][d] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    if (threadIdx.x < 3)
      for (int wi = 0; wi < kReduceThreads / 32; ++wi) v += red[wi][threadIdx.x];
    part[4 * blockIdx.x + threadIdx.x] = v;
  }
}

__global__ void __launch_bounds__(kReduceThreads) k_field_sum_final(const double* part, int nparts,
                                                                    int D, double* out) {
  if (threadIdx.x < 3) {
    double s = 0;
    for (int i = 0; i < nparts; ++i) s += part[4 * i + threadIdx.x];
    if (static_cast<int>(threadIdx.x) < D) out[threadIdx.x] = s;
  }
}

}  // namespace lbm
