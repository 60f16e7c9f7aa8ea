// Payload of a streaming frame (MADDENING BinaryStateEncoder.encode,
// src/maddening/api/binary_encoder.py:151-205): device arrays converted to
// float32 and laid end to end, every field of one frame in one launch
// (blockIdx.y = field, a grid-stride loop over its elements).  Conversions
// round to nearest like NumPy's astype(float32).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace lbm {

constexpr int kPackMaxFields = 32;
constexpr int kPackThreads = 256;

enum PackType : int32_t {
  kPackF32 = 0, kPackF16 = 1, kPackBF16 = 2, kPackF64 = 3, kPackU8 = 4, kPackI32 = 5,
  kPackI64 = 6
};

struct PackBatch {
  const void* src[kPackMaxFields];
  int64_t count[kPackMaxFields];
  int64_t offset[kPackMaxFields];  // first element in the payload
  int32_t type[kPackMaxFields];
};

__device__ __forceinline__ float pack_value(const void* p, int32_t type, int64_t i) {
  switch (type) {
    case kPackF16: return __half2float(static_cast<const __half*>(p)[i]);
    case kPackBF16: return __bfloat162float(static_cast<const __nv_bfloat16*>(p)[i]);
    case kPackF64: return __double2float_rn(static_cast<const double*>(p)[i]);
    case kPackU8: return static_cast<float>(static_cast<const uint8_t*>(p)[i]);
    case kPackI32: return __int2float_rn(static_cast<const int32_t*>(p)[i]);
    case kPackI64: return __ll2float_rn(static_cast<const long long*>(p)[i]);
    default: return static_cast<const float*>(p)[i];
  }
}

__global__ void __launch_bounds__(kPackThreads) k_pack_f32(const __grid_constant__ PackBatch b,
                                                           float* out) {
  const int f = blockIdx.y;
  const void* src = b.src[f];
  const int64_t n = b.count[f];
  const int32_t type = b.type[f];
  float* dst = out + b.offset[f];
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kPackThreads;
  int64_t i = static_cast<int64_t>(blockIdx.x) * kPackThreads + threadIdx.x;
  // four independent loads in flight per thread, then the remainder
  for (; i + 3 * stride < n; i += 4 * stride) {
    const float v0 = pack_value(src, type, i);
    const float v1 = pack_value(src, type, i + stride);
    const float v2 = pack_value(src, type, i + 2 * stride);
    const float v3 = pack_value(src, type, i + 3 * stride);
    dst[i] = v0;
    dst[i + stride] = v1;
    dst[i + 2 * stride] = v2;
    dst[i + 3 * stride] = v3;
  }
  for (; i < n; i += stride) dst[i] = pack_value(src, type, i);
}

}  // namespace lbm
