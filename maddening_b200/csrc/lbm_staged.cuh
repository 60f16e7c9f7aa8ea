// Row-staged fused step: the pull's neighbour rows are moved into shared
// memory by the copy engine (1-D bulk asynchronous copies, cp.async.bulk,
// completion tracked by an mbarrier), so threads read their 19 populations
// from shared memory instead of computing 19 global addresses each.
//
// A persistent CTA walks whole rows (i0, i1) of the lattice with a grid
// stride.  For row r it needs, for every direction q, the full source row
// (i0 - c0, i1 - c1) of plane q (the shift -c2 along the row is applied when
// reading shared memory, with the periodic wrap).  One thread arms the stage's
// mbarrier with the expected byte count and issues the Q copies; a ring of
// `stages` buffers keeps stages-1 rows in flight while the current row is
// computed.  Every wait is bounded: on timeout the CTA records the failure in
// *status, waits (bounded) for its own copies still in flight and returns.
//
// Requirements (checked on the host): row bytes n2 * sizeof(S) a multiple of
// 16 (bulk-copy alignment of source, destination and size), rows short enough
// for `stages` row sets in shared memory.  Used for the state-to-state steps
// of a rollout; the other modes keep the global-memory gather.
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (bulk copy) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Global -> this CTA's shared memory, `bytes` a multiple of 16, both addresses
// 16-byte aligned; completion is signalled on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait suspends for a hardware-chosen interval per call; 2^22 calls are
// far beyond any copy's latency, and still end.
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// This CTA's shared memory -> global, `bytes` a multiple of 16, both addresses
// 16-byte aligned; tracked in the issuing thread's bulk async-group, which
// this call commits.
__device__ __forceinline__ void bulk_store_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// The issuing thread's bulk stores have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// The issuing thread's bulk stores are complete.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// 1024 resident threads per SM (<= 64 registers) for 32-bit arithmetic, 512
// for FP64.
template <class S, int T>
constexpr int staged_min_blocks() {
  return (sizeof(typename StoreT<S>::R) == 8 ? 512 : 1024) / T;
}

template <int Q, class S, bool FACES, bool FORCE, int T>
__global__ void __launch_bounds__(T, staged_min_blocks<S, T>())
    k_step_staged(const __grid_constant__ StepArgs a, int stages) {
  using R = typename StoreT<S>::R;
  extern __shared__ __align__(128) unsigned char smem[];
  const Geo& g = a.g;
  const uint32_t row_bytes = g.n2 * static_cast<uint32_t>(sizeof(S));
  const uint32_t stage_bytes = static_cast<uint32_t>(Q) * row_bytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + static_cast<size_t>(stages) * stage_bytes);
  const uint32_t nrows = g.n0 * g.n1;
  const uint32_t G = gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Thread 0: arm stage s and copy the Q source rows of lattice row `row`.
  auto issue = [&](uint32_t row, int s) {
    const uint32_t i0 = fdiv(row, g.div_n1);
    const uint32_t i1 = row - i0 * g.n1;
    const uint32_t r0m = i0 == 0 ? g.n0 - 1 : i0 - 1, r0p = i0 == g.n0 - 1 ? 0 : i0 + 1;
    const uint32_t r1m = i1 == 0 ? g.n1 - 1 : i1 - 1, r1p = i1 == g.n1 - 1 ? 0 : i1 + 1;
    unsigned char* dst = smem + static_cast<size_t>(s) * stage_bytes;
    mbar_arrive_expect_tx(&bars[s], stage_bytes);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int c0 = Lat<Q>::c0(q), c1 = Lat<Q>::c1(q);
      const uint32_t j0 = c0 > 0 ? r0m : (c0 < 0 ? r0p : i0);
      const uint32_t j1 = c1 > 0 ? r1m : (c1 < 0 ? r1p : i1);
      const S* src = static_cast<const S*>(a.pin) +
                     (static_cast<uint32_t>(q) * g.pstride + (j0 * g.n1 + j1) * g.rstride);
      bulk_copy_g2s(dst + static_cast<size_t>(q) * row_bytes, src, row_bytes, &bars[s]);
    }
  };

  if (threadIdx.x == 0) {
    for (int j = 0; j < stages - 1; ++j) {
      const uint32_t row = blockIdx.x + static_cast<uint32_t>(j) * G;
      if (row < nrows) issue(row, j);
    }
  }

  bool failed = false;
  uint32_t it = 0;
  for (uint32_t row = blockIdx.x; row < nrows; row += G, ++it) {
    const int s = static_cast<int>(it % static_cast<uint32_t>(stages));
    if (threadIdx.x == 0) {
      // Prefetch into the stage consumed in the previous iteration (every
      // thread passed that iteration's closing barrier).
      const uint32_t pr = row + static_cast<uint32_t>(stages - 1) * G;
      if (pr < nrows) {
        fence_proxy_async_smem();
        issue(pr, static_cast<int>((it + stages - 1) % static_cast<uint32_t>(stages)));
      }
    }
    const bool ok = mbar_wait_bounded(&bars[s], (it / static_cast<uint32_t>(stages)) & 1u);
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    const S* buf = reinterpret_cast<const S*>(smem + static_cast<size_t>(s) * stage_bytes);
    Cell x;
    x.i0 = fdiv(row, g.div_n1);
    x.i1 = row - x.i0 * g.n1;
    x.row = row * g.n2;
    x.srow = row * g.rstride;
    for (uint32_t k = threadIdx.x; k < g.n2; k += T) {
      x.k = k;
      x.c = x.row + k;
      const uint32_t km = k == 0 ? g.n2 - 1 : k - 1;
      const uint32_t kp = k == g.n2 - 1 ? 0 : k + 1;
      R d[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int c2 = Lat<Q>::c2(q);
        const uint32_t kk = c2 > 0 ? km : (c2 < 0 ? kp : k);
        d[q] = to_r(buf[static_cast<uint32_t>(q) * g.n2 + kk]);
      }
      finish_cell<Q, S, kOutState, FACES, FORCE>(a, x, d);
    }
    __syncthreads();  // stage s fully read before it is refilled
  }
  if (failed && threadIdx.x == 0) {
    atomicOr(a.status, 1);
    // Let the copies this CTA issued and has not waited for land before it
    // exits: rows of iterations it .. it + stages - 1 (bounded waits).
    for (uint32_t j = it; j < it + static_cast<uint32_t>(stages); ++j) {
      if (blockIdx.x + j * G >= nrows) break;
      (void)mbar_wait_bounded(&bars[j % static_cast<uint32_t>(stages)],
                              (j / static_cast<uint32_t>(stages)) & 1u);
    }
  }
}

}  // namespace lbm
