// Launchers of the one-pass tiled step (lbm_tiled.cuh), in a translation unit
// of their own so that the library's units compile in parallel.
#include <algorithm>

#include "lbm_host.h"
#include "lbm_tiled.cuh"

namespace {

// Sweep geometry and work items for a persistent grid of `grid` blocks: the
// number of chunks along the sweep axis minimises the planes of the busiest
// block, ceil(items / grid) x (planes per chunk + 2 halo planes).
template <int Q>
lbm::TileGeo tile_geo(const lbm_plan* p, uint32_t grid) {
  using T = lbm::TileShape<Q>;
  lbm::TileGeo t{};
  const lbm::Geo& g = p->g;
  if (Q == 19) {
    t.NS = g.n0; t.NR = g.n1; t.SS = g.n1 * g.n2; t.SR = g.n2;
  } else {
    t.NS = g.n1; t.NR = 1; t.SS = g.n2; t.SR = 0;
  }
  t.ncolz = (g.n2 + T::TZ - 1) / T::TZ;
  t.ncol = t.ncolz * ((t.NR + T::TY - 1) / T::TY);
  uint64_t best = ~uint64_t(0);
  uint32_t best_chunk = t.NS;
  const uint32_t kmax = std::min<uint32_t>(t.NS, 4096);
  for (uint32_t k = 1; k <= kmax; ++k) {
    const uint32_t chunk = (t.NS + k - 1) / k;
    const uint64_t nch = (t.NS + chunk - 1) / chunk;
    const uint64_t items = nch * t.ncol;
    const uint64_t cost = ((items + grid - 1) / grid) * (chunk + 2);
    if (cost < best) { best = cost; best_chunk = chunk; }
  }
  t.chunk = best_chunk;
  t.items = t.ncol * ((t.NS + best_chunk - 1) / best_chunk);
  // a copy or a neighbouring warp takes microseconds; 2 s means something broke
  const bool test = (p->flags & LBM_PLAN_TEST_WAIT_TIMEOUT) != 0;
  t.wait_ns = test ? 200000ull : 2000000000ull;
  t.no_copy = test ? 1u : 0u;
  return t;
}

template <int Q, class S, int MODE, bool FACES, bool FORCE>
int launch_tiled_t(const lbm_plan* p, const lbm::StepArgs& a, cudaStream_t s) {
  auto kern = lbm::k_tiled<Q, S, MODE, FACES, FORCE>;
  constexpr size_t smem = lbm::tiled_smem_bytes<Q, MODE>();
  int rc = cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem)),
                      "cudaFuncSetAttribute");
  if (rc) return rc;
  int dev = 0, sms = 148, per_sm = 0;
  rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  rc = cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                  "cudaDeviceGetAttribute");
  if (rc) return rc;
  rc = cuda_check(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, lbm::TileShape<Q>::NT, smem),
      "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (rc) return rc;
  if (per_sm < 1) return fail(LBM_ERR_CUDA, "tiled step: no resident block (%zu B smem)", smem);
  const uint32_t grid = static_cast<uint32_t>(per_sm) * static_cast<uint32_t>(sms);
  const lbm::TileGeo t = tile_geo<Q>(p, grid);
  kern<<<std::min(grid, t.items), lbm::TileShape<Q>::NT, smem, s>>>(a, t);
  return cuda_check(cudaGetLastError(), "k_tiled launch");
}

}  // namespace

template <int Q, class S, int MODE>
int launch_tiled(const lbm_plan* p, const lbm::StepArgs& a, cudaStream_t s) {
  const bool faces = a.face[0].kind != lbm::kFaceNone || a.face[1].kind != lbm::kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) return force ? launch_tiled_t<Q, S, MODE, true, true>(p, a, s)
                          : launch_tiled_t<Q, S, MODE, true, false>(p, a, s);
  return force ? launch_tiled_t<Q, S, MODE, false, true>(p, a, s)
               : launch_tiled_t<Q, S, MODE, false, false>(p, a, s);
}

#define LBM_TILED_INST(Q, S)                                                             \
  template int launch_tiled<Q, S, lbm::kOutAoS>(const lbm_plan*, const lbm::StepArgs&,   \
                                                cudaStream_t);                           \
  template int launch_tiled<Q, S, lbm::kOutState>(const lbm_plan*, const lbm::StepArgs&, \
                                                  cudaStream_t);
LBM_TILED_INST(19, float)
LBM_TILED_INST(19, __half)
LBM_TILED_INST(19, __nv_bfloat16)
LBM_TILED_INST(9, float)
LBM_TILED_INST(9, __half)
LBM_TILED_INST(9, __nv_bfloat16)
