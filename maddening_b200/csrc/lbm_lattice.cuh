// Compile-time lattice constants for the D3Q19 and D2Q9 velocity sets.
//
// Direction order follows the reference (d3q19: src/maddening/nodes/lbm.py:92-135,
// d2q9: lbm.py:144-169), because the (*grid_shape, Q) state layout depends on it.
//
// Kernels address a lattice as three internal axes (a0, a1, a2) with a2
// contiguous in memory.  A 3-D grid_shape (n0, n1, n2) maps 1:1; a 2-D grid
// (nx, ny) is the single plane (1, nx, ny), so D2Q9 directions carry a zero
// a0 component and reference axis d maps to internal axis d + (3 - D).
#pragma once

#include <cstdint>

namespace lbm {

template <int Q>
struct Lat;

template <>
struct Lat<19> {
  static constexpr int D = 3;
  __host__ __device__ static constexpr int c0(int q) {
    constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[q];
  }
  __host__ __device__ static constexpr int c1(int q) {
    constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int c2(int q) {
    constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int opp(int q) {
    constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    return t[q];
  }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
  }
  // w(q) = wr(q) / kWDen with integer wr
  static constexpr int kWDen = 36;
  __host__ __device__ static constexpr int wr(int q) { return q == 0 ? 12 : (q <= 6 ? 2 : 1); }
};

template <>
struct Lat<9> {
  static constexpr int D = 2;
  __host__ __device__ static constexpr int c0(int) { return 0; }
  __host__ __device__ static constexpr int c1(int q) {
    constexpr int t[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int c2(int q) {
    constexpr int t[9] = {0, 0, 0, 1, -1, 1, 1, -1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int opp(int q) {
    constexpr int t[9] = {0, 2, 1, 4, 3, 8, 7, 6, 5};
    return t[q];
  }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 4.0 / 9.0 : (q <= 4 ? 1.0 / 9.0 : 1.0 / 36.0);
  }
  static constexpr int kWDen = 36;
  __host__ __device__ static constexpr int wr(int q) { return q == 0 ? 16 : (q <= 4 ? 4 : 1); }
};

// Component of direction q along internal axis a (a is a runtime value).
template <int Q>
__host__ __device__ constexpr int comp(int q, int a) {
  return a == 0 ? Lat<Q>::c0(q) : (a == 1 ? Lat<Q>::c1(q) : Lat<Q>::c2(q));
}

// w split into a float head and a float tail: w == w_hi + w_lo to ~1e-16.
// f32 offsets are exact w.r.t. the true weight: g = (f - w_hi) - w_lo.
template <int Q>
__host__ __device__ constexpr float w_hi(int q) {
  return static_cast<float>(Lat<Q>::w(q));
}
template <int Q>
__host__ __device__ constexpr float w_lo(int q) {
  return static_cast<float>(Lat<Q>::w(q) - static_cast<double>(w_hi<Q>(q)));
}

}  // namespace lbm
