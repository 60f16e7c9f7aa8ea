// Host-side pieces shared by the translation units of liblbm_b200.so: the plan,
// the error helpers behind lbm_last_error, and the launchers that live in
// their own units (compiled in parallel).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lbm_b200.h"
#include "lbm_kernels.cuh"

struct lbm_plan {
  int Q = 0, D = 0, storage = 0;
  int64_t shape[3] = {0, 0, 0};  // reference grid_shape
  lbm::Geo g{};                  // internal geometry
  double tau = 0;
  size_t elem = 4;               // bytes per stored population
  size_t io = 4;                 // bytes per f / force / moment element
  uint32_t flags = 0;            // LBM_PLAN_* bits
};

// Records the message for lbm_last_error (calling thread) and returns code.
int fail(int code, const char* fmt, ...);
// LBM_OK, or fail(LBM_ERR_CUDA, "<what>: <CUDA message>").
int cuda_check(cudaError_t e, const char* what);

// One-pass tiled step (lbm_tiled.cuh, launched from lbm_tiled.cu) for 32-bit
// IO: MODE lbm::kOutAoS (a whole update) or lbm::kOutState (the first step of a
// rollout).  Instantiated for Q in {9, 19}, S in {float, __half, __nv_bfloat16}.
template <int Q, class S, int MODE>
int launch_tiled(const lbm_plan* p, const lbm::StepArgs& a, cudaStream_t s);
