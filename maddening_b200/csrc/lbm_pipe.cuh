// D3Q7 passive tracer of the pipe node (MADDENING LBMPipeNode.update, tracer
// branch, src/maddening/nodes/lbm_pipe.py:857-871):
//   tracer = sum g;  g_eq_q = w7_q tracer (1 + e_q.u / cs2)   (u: this step's
//   new velocity, 0 in walls);  g_post = g in walls, else g - (g - g_eq)/tau_t;
//   g_str = periodic shift by e_q;  g_bc = where(wall, g_str[opp], g_str);
//   tracer_out = sum g_bc (0 in walls).
// The collision needs the velocity of the same step at the same cell: the
// D3Q19 pull step has it in registers once it has taken the moments of f_bc,
// so k_pipe_step runs the tracer of the cell in the same thread, in push
// form: the cell collides its own populations and sends population q to
// y = x + e_q, into slot opp(q) when y is a wall (the wall swap taken at the
// destination; every slot is written exactly once).  Populations are FP32
// (FP64 with FP64 plans), one plane per direction.
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

struct Lat7 {
  __host__ __device__ static constexpr int c(int q, int a) {
    // rest, +x, -x, +y, -y, +z, -z (the first seven D3Q19 directions)
    return q == 0 ? 0 : ((q - 1) / 2 == a ? ((q & 1) ? 1 : -1) : 0);
  }
  __host__ __device__ static constexpr int opp(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
  __host__ __device__ static constexpr double w(int q) { return q == 0 ? 0.25 : 0.125; }
};

struct TracerArgs {
  Geo g;
  const uint8_t* wall;
  const void* tin;      // populations (7 planes)
  void* tout;
  double inv_tau;       // 1 / tau_tracer
  const void* f7_in;    // (grid, 7) reference layout (prepare)
  void* f7_out;         // (grid, 7) reference layout (final)
  void* tracer_out;     // grid (final)
};

template <class IO>
__global__ void __launch_bounds__(kBlock) k_tracer_prepare(const TracerArgs a) {
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  const IO* fi = aos_fill<7, IO>(static_cast<const IO*>(a.f7_in), blockIdx.x * kBlock, a.g.ncell);
  if (c >= a.g.ncell) return;
#pragma unroll
  for (int q = 0; q < 7; ++q) static_cast<IO*>(a.tout)[static_cast<size_t>(q) * a.g.ncell + c] = fi[q];
}

// Tracer step of cell x with this step's velocity uu (0 in walls).
template <class IO>
__device__ __forceinline__ void tracer_cell(const TracerArgs& a, const Cell& x, bool wall,
                                            const IO (&uu)[3]) {
  const Geo& g = a.g;
  const uint32_t c = x.c;
  const IO* tin = static_cast<const IO*>(a.tin);
  IO t[7];
#pragma unroll
  for (int q = 0; q < 7; ++q) t[q] = tin[static_cast<size_t>(q) * g.ncell + c];
  if (!wall) {
    IO tracer = t[0];
#pragma unroll
    for (int q = 1; q < 7; ++q) tracer = add_r(tracer, t[q]);
    const IO it = static_cast<IO>(a.inv_tau);
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      IO eu = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (Lat7::c(q, d)) eu = Lat7::c(q, d) > 0 ? uu[d] : -uu[d];
      const IO geq = mul_r(mul_r(static_cast<IO>(Lat7::w(q)), tracer), fma_r(IO(3), eu, IO(1)));
      t[q] = fma_r(-it, sub_r(t[q], geq), t[q]);
    }
  }
  IO* tout = static_cast<IO*>(a.tout);
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    const uint32_t j0 = wrapu(static_cast<int>(x.i0) + Lat7::c(q, 0), g.n0);
    const uint32_t j1 = wrapu(static_cast<int>(x.i1) + Lat7::c(q, 1), g.n1);
    const uint32_t j2 = wrapu(static_cast<int>(x.k) + Lat7::c(q, 2), g.n2);
    const uint32_t y = (j0 * g.n1 + j1) * g.n2 + j2;
    const bool wy = a.wall != nullptr && a.wall[y] != 0;
    const int slot = wy ? Lat7::opp(q) : q;
    tout[static_cast<size_t>(slot) * g.ncell + y] = t[q];
  }
}

// One pipe-node step of cell x: the D3Q19 pull step with the pipe force
// (force mode 3: no half-force step in the moments), then the tracer step of
// the same cell with the velocity just taken (lbm_pipe.py:751-879).  LAST
// writes f_bc in the reference layout and the moment outputs instead of
// colliding.
template <class S, bool LAST>
__global__ void __launch_bounds__(kBlock, min_blocks<S>())
    k_pipe_step(const __grid_constant__ StepArgs a, const __grid_constant__ TracerArgs t) {
  using R = typename StoreT<S>::R;
  using IO = typename StoreT<S>::IO;
  const uint32_t cidx = blockIdx.x * kBlock + threadIdx.x;
  if (cidx < a.g.ncell) {
    const Cell x = locate(a.g, cidx);
    R d[19];
    pull_cell<19, S>(a, x, d);
    const bool wall = a.wall != nullptr && __ldg(a.wall + cidx) != 0;
    R F[3];
    pipe_force<R>(a, cidx, wall, F);
    apply_bc<19, S, false>(a, x, wall, d);
    const Mom<R> m = moments<19, R, true>(d, F, false);
    if (LAST) {
      store_moments<19, IO>(a, cidx, m, wall);
      IO* row = aos_tile<19, IO>() + threadIdx.x * 19;
#pragma unroll
      for (int q = 0; q < 19; ++q) row[q] = static_cast<IO>(from_offset<19, R>(d[q], q));
    } else {
      collide<19, R, true>(d, m, F, static_cast<R>(a.omega), static_cast<R>(a.guo_c));
#pragma unroll
      for (int q = 0; q < 19; ++q)
        static_cast<S*>(a.pout)[static_cast<uint32_t>(q) * a.g.pstride + x.srow + x.k] =
            from_r<S>(d[q]);
    }
    const IO uu[3] = {wall ? IO(0) : static_cast<IO>(m.u[0]),
                      wall ? IO(0) : static_cast<IO>(m.u[1]),
                      wall ? IO(0) : static_cast<IO>(m.u[2])};
    tracer_cell<IO>(t, x, wall, uu);
  }
  if (LAST) aos_flush<19, IO>(static_cast<IO*>(a.f_out), blockIdx.x * kBlock, a.g.ncell);
}

// Last pass: populations to the reference layout and the tracer field.
template <class IO>
__global__ void __launch_bounds__(kBlock) k_tracer_final(const TracerArgs a) {
  const uint32_t c = blockIdx.x * kBlock + threadIdx.x;
  if (c < a.g.ncell) {
    const IO* tin = static_cast<const IO*>(a.tin);
    IO* row = aos_tile<7, IO>() + threadIdx.x * 7;
    IO s = 0;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      const IO v = tin[static_cast<size_t>(q) * a.g.ncell + c];
      row[q] = v;
      s = q == 0 ? v : add_r(s, v);
    }
    if (a.tracer_out != nullptr) {
      const bool wall = a.wall != nullptr && a.wall[c] != 0;
      static_cast<IO*>(a.tracer_out)[c] = wall ? IO(0) : s;
    }
  }
  aos_flush<7, IO>(static_cast<IO*>(a.f7_out), blockIdx.x * kBlock, a.g.ncell);
}

}  // namespace lbm
