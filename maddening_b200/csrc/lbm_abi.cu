// C ABI of the lattice-Boltzmann node step: plan validation, argument
// mapping and kernel dispatch.  Declarations and contracts: include/lbm_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_adjoint.cuh"
#include "lbm_kernels.cuh"
#include "lbm_pair.cuh"
#include "lbm_multiphase.cuh"
#include "lbm_pack.cuh"
#include "lbm_pipe.cuh"
#include "lbm_staged.cuh"
#include "lbm_host.h"

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return fail(LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return LBM_OK;
}

namespace {

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

size_t state_bytes(const lbm_plan* p) {
  return static_cast<size_t>(p->Q) * static_cast<size_t>(p->g.ncell) * p->elem;
}

// Multiply-high constants for x / d, 0 <= x < 2^31 (see lbm::fdiv).
lbm::FastDiv make_fastdiv(uint32_t d) {
  lbm::FastDiv f;
  f.d = d;
  uint32_t s = 0;
  while ((uint64_t(1) << s) < d) ++s;
  f.s = s;
  f.m = static_cast<uint32_t>(((uint64_t(1) << 32) * ((uint64_t(1) << s) - d)) / d + 1);
  return f;
}

uint32_t host_fdiv(uint32_t x, const lbm::FastDiv& f) {
  const uint32_t hi = static_cast<uint32_t>((static_cast<uint64_t>(x) * f.m) >> 32);
  return (hi + x) >> f.s;
}

bool fastdiv_ok(const lbm::FastDiv& f, uint32_t xmax) {
  const uint32_t probes[] = {0u, 1u, f.d - 1, f.d, f.d + 1, 2 * f.d - 1, 2 * f.d,
                             xmax / 2, xmax - 1, xmax};
  for (uint32_t x : probes)
    if (x <= xmax && host_fdiv(x, f) != x / f.d) return false;
  return true;
}



// Maps one face condition of the ABI to the kernel form (internal axes).
int map_face(const lbm_plan* p, const lbm_face_bc& in, bool is_outlet, lbm::FaceK* out) {
  std::memset(out, 0, sizeof(*out));
  out->kind = lbm::kFaceNone;
  if (in.kind == LBM_BC_NONE) return LBM_OK;
  if (in.kind < LBM_BC_NONE || in.kind > LBM_BC_ZERO_GRADIENT)
    return fail(LBM_ERR_INVALID, "unknown face condition kind %d", in.kind);
  if (in.face < LBM_FACE_X_MIN || in.face > LBM_FACE_Z_MAX)
    return fail(LBM_ERR_INVALID, "unknown face %d", in.face);
  const int ref_axis = in.face / 2;
  if (ref_axis >= p->D)
    return fail(LBM_ERR_INVALID,
                "face %d uses axis %d but lattice D%dQ%d only has %d dimensions", in.face,
                ref_axis, p->D, p->Q, p->D);
  const int sh = 3 - p->D;
  out->kind = in.kind;
  out->ref_axis = ref_axis;
  out->axis = ref_axis + sh;
  out->side = in.face % 2;
  if (in.kind == LBM_BC_PRESSURE) {
    out->v[0] = in.value[0];
  } else if (in.kind == LBM_BC_VELOCITY) {
    for (int d = 0; d < p->D; ++d) out->v[d + sh] = in.value[d];
  } else if (in.kind == LBM_BC_ZERO_GRADIENT) {
    if (!is_outlet) return fail(LBM_ERR_INVALID, "zero-gradient is an outlet condition");
    if (p->shape[ref_axis] < 3)
      return fail(LBM_ERR_INVALID, "zero-gradient face needs >= 3 cells along axis %d",
                  ref_axis);
  }
  return LBM_OK;
}

int build_args(const lbm_plan* p, const lbm_step_args* args, const lbm_moments* mom,
               lbm::StepArgs* a) {
  std::memset(a, 0, sizeof(*a));
  a->g = p->g;
  a->cell0 = 0;
  a->cell_end = p->g.ncell;
  a->omega = 1.0 / p->tau;
  a->guo_c = 1.0 - 0.5 / p->tau;
  if (args == nullptr) return fail(LBM_ERR_INVALID, "args is NULL");
  a->force_mode = args->force_mode;
  const int sh = 3 - p->D;
  if (args->force_mode == LBM_FORCE_UNIFORM) {
    for (int d = 0; d < p->D; ++d) a->force[d + sh] = args->force[d];
  } else if (args->force_mode == LBM_FORCE_FIELD) {
    if (args->force_field == nullptr)
      return fail(LBM_ERR_INVALID, "force_mode FIELD needs force_field");
    a->force_field = args->force_field;
  } else if (args->force_mode != LBM_FORCE_NONE) {
    return fail(LBM_ERR_INVALID, "unknown force_mode %d", args->force_mode);
  }
  a->wall = args->wall;
  int rc = map_face(p, args->inlet, false, &a->face[0]);
  if (rc) return rc;
  rc = map_face(p, args->outlet, true, &a->face[1]);
  if (rc) return rc;
  if (a->face[1].kind == lbm::kFaceZeroGrad && a->face[0].kind != lbm::kFaceNone &&
      a->face[0].axis != a->face[1].axis)
    return fail(LBM_ERR_UNSUPPORTED,
                "a zero-gradient outlet needs the inlet on the same axis (or no inlet)");
  a->dev_values = args->dev_values;
  if (mom != nullptr) {
    a->rho = mom->density;
    a->vel = mom->velocity;
    a->prs = mom->pressure;
    a->mflags = mom->flags;
  }
  return LBM_OK;
}

unsigned grid_for(uint64_t n) { return static_cast<unsigned>((n + lbm::kBlock - 1) / lbm::kBlock); }

template <int Q, class S>
int launch_prepare(const lbm::StepArgs& a, cudaStream_t s) {
  const unsigned grid = grid_for(a.g.ncell);
  if (a.force_mode != 0)
    lbm::k_prepare<Q, S, true><<<grid, lbm::kBlock, 0, s>>>(a);
  else
    lbm::k_prepare<Q, S, false><<<grid, lbm::kBlock, 0, s>>>(a);
  return cuda_check(cudaGetLastError(), "k_prepare launch");
}

template <int Q, class S, int MODE>
void launch_step_mode(const lbm::StepArgs& a, cudaStream_t s) {
  const unsigned grid = grid_for(a.cell_end - a.cell0);
  const bool faces = a.face[0].kind != lbm::kFaceNone || a.face[1].kind != lbm::kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) {
    if (force) lbm::k_step<Q, S, MODE, true, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step<Q, S, MODE, true, false><<<grid, lbm::kBlock, 0, s>>>(a);
  } else {
    if (force) lbm::k_step<Q, S, MODE, false, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step<Q, S, MODE, false, false><<<grid, lbm::kBlock, 0, s>>>(a);
  }
}

template <int Q, class S>
int launch_step(const lbm::StepArgs& a, bool final_aos, cudaStream_t s) {
  if (final_aos) launch_step_mode<Q, S, lbm::kOutAoS>(a, s);
  else launch_step_mode<Q, S, lbm::kOutState>(a, s);
  return cuda_check(cudaGetLastError(), "k_step launch");
}

// Paired-cell state step (lbm_pair.cuh): the default for 16-bit storage,
// opt-in for FP32 (LBM_PLAN_PAIRED_CELLS), off with LBM_PLAN_SINGLE_CELLS.
// Rows of even length (row segments when they split into warps of 64 cells,
// instance-wide pairs otherwise); state planes and the wall mask aligned for
// the pair width.
template <class S>
bool pair_ok(const lbm_plan* p, const lbm::StepArgs& a) {
  if constexpr (sizeof(S) == 8) {
    return false;
  } else {
    if (p->flags & LBM_PLAN_SINGLE_CELLS) return false;
    if (sizeof(S) == 4 && !(p->flags & LBM_PLAN_PAIRED_CELLS)) return false;
    const uintptr_t al = 2 * sizeof(S);
    return p->g.n2 % 2 == 0 && reinterpret_cast<uintptr_t>(a.pin) % al == 0 &&
           reinterpret_cast<uintptr_t>(a.pout) % al == 0 &&
           reinterpret_cast<uintptr_t>(a.wall) % 2 == 0;
  }
}

template <int Q, class S, int W>
void launch_pair_w(const lbm::StepArgs& a, cudaStream_t s) {
  const dim3 grid(a.g.n0 * a.g.n1, a.g.n2 / (64 * W));
  const bool faces = a.face[0].kind != lbm::kFaceNone || a.face[1].kind != lbm::kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) {
    if (force) lbm::k_step_pair<Q, S, true, true, W><<<grid, 32 * W, 0, s>>>(a);
    else lbm::k_step_pair<Q, S, true, false, W><<<grid, 32 * W, 0, s>>>(a);
  } else {
    if (force) lbm::k_step_pair<Q, S, false, true, W><<<grid, 32 * W, 0, s>>>(a);
    else lbm::k_step_pair<Q, S, false, false, W><<<grid, 32 * W, 0, s>>>(a);
  }
}

template <int Q, class S, int W>
void launch_quad_w(const lbm::StepArgs& a, cudaStream_t s) {
  const dim3 grid(a.g.n0 * a.g.n1, a.g.n2 / (128 * W));
  const bool faces = a.face[0].kind != lbm::kFaceNone || a.face[1].kind != lbm::kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) {
    if (force) lbm::k_step_quad<Q, S, true, true, W><<<grid, 32 * W, 0, s>>>(a);
    else lbm::k_step_quad<Q, S, true, false, W><<<grid, 32 * W, 0, s>>>(a);
  } else {
    if (force) lbm::k_step_quad<Q, S, false, true, W><<<grid, 32 * W, 0, s>>>(a);
    else lbm::k_step_quad<Q, S, false, false, W><<<grid, 32 * W, 0, s>>>(a);
  }
}

// The four-cell form (16-bit storage): rows of a multiple of 128 cells,
// unpadded state rows, 8-byte aligned planes and a 4-byte aligned wall mask.
// D3Q19 also takes it (a B200 sweep at 256^3: 79.2k MLUPS FP16 against 71.7k
// for pairs, at 20 resident warps and 96 registers) on rows of a multiple of
// 256 cells: with one-warp blocks (rows of 128) it keeps 15 warps resident and
// loses to pairs.
#ifndef LBM_QUAD_Q19
#define LBM_QUAD_Q19 1
#endif
template <int Q, class S>
bool quad_ok(const lbm::StepArgs& a) {
  return (Q == 9 || (LBM_QUAD_Q19 && Q == 19)) && sizeof(S) == 2 &&
         a.g.n2 % (Q == 19 ? 256 : 128) == 0 && a.g.rstride == a.g.n2 &&
         a.g.pstride % 4 == 0 && reinterpret_cast<uintptr_t>(a.pin) % 8 == 0 &&
         reinterpret_cast<uintptr_t>(a.pout) % 8 == 0 &&
         reinterpret_cast<uintptr_t>(a.wall) % 4 == 0;
}

template <int Q, class S>
void launch_gquad(const lbm::StepArgs& a, cudaStream_t s) {
  const unsigned grid = grid_for(a.g.ncell / 4);
  const bool faces = a.face[0].kind != lbm::kFaceNone || a.face[1].kind != lbm::kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) {
    if (force) lbm::k_step_gquad<Q, S, true, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step_gquad<Q, S, true, false><<<grid, lbm::kBlock, 0, s>>>(a);
  } else {
    if (force) lbm::k_step_gquad<Q, S, false, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step_gquad<Q, S, false, false><<<grid, lbm::kBlock, 0, s>>>(a);
  }
}

// The instance-wide four-cell form: D2Q9 with 16-bit storage, rows of a
// multiple of 4 cells (a quad never spans two rows), the same alignment as the
// row form (4000^2 channel: 148.9k MLUPS against 114.4k for pairs).  D3Q19
// keeps pairs there: with per-lane rows its 96-register budget spills and it
// lost (48.3k against 61.9k at 160^3; 56.4k at 128 registers and 16 warps).
template <int Q, class S>
bool gquad_ok(const lbm::StepArgs& a) {
  return Q == 9 && sizeof(S) == 2 && a.g.n2 % 4 == 0 &&
         a.g.rstride == a.g.n2 && a.g.pstride % 4 == 0 &&
         reinterpret_cast<uintptr_t>(a.pin) % 8 == 0 &&
         reinterpret_cast<uintptr_t>(a.pout) % 8 == 0 &&
         reinterpret_cast<uintptr_t>(a.wall) % 4 == 0;
}

template <int Q, class S>
void launch_gpair(const lbm::StepArgs& a, cudaStream_t s) {
  const unsigned grid = grid_for(a.g.ncell / 2);
  const bool faces = a.face[0].kind != lbm::kFaceNone || a.face[1].kind != lbm::kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) {
    if (force) lbm::k_step_gpair<Q, S, true, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step_gpair<Q, S, true, false><<<grid, lbm::kBlock, 0, s>>>(a);
  } else {
    if (force) lbm::k_step_gpair<Q, S, false, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step_gpair<Q, S, false, false><<<grid, lbm::kBlock, 0, s>>>(a);
  }
}

template <int Q, class S>
int launch_pair(const lbm::StepArgs& a, cudaStream_t s) {
  if constexpr (sizeof(S) == 8) {
    return fail(LBM_ERR_UNSUPPORTED, "paired step has no FP64 form");
  } else {
    if constexpr ((Q == 9 || (LBM_QUAD_Q19 && Q == 19)) && sizeof(S) == 2) {
      if (quad_ok<Q, S>(a)) {
        if (a.g.n2 % 512 == 0) launch_quad_w<Q, S, 4>(a, s);
        else if (a.g.n2 % 256 == 0) launch_quad_w<Q, S, 2>(a, s);
        else launch_quad_w<Q, S, 1>(a, s);
        return cuda_check(cudaGetLastError(), "k_step_quad launch");
      }
    }
    if constexpr (Q == 9 && sizeof(S) == 2) {
      if (gquad_ok<Q, S>(a)) {
        launch_gquad<Q, S>(a, s);
        return cuda_check(cudaGetLastError(), "k_step_gquad launch");
      }
    }
    if (a.g.n2 % 256 == 0) launch_pair_w<Q, S, 4>(a, s);
    else if (a.g.n2 % 128 == 0) launch_pair_w<Q, S, 2>(a, s);
    else if (a.g.n2 % 64 == 0) launch_pair_w<Q, S, 1>(a, s);
    else launch_gpair<Q, S>(a, s);
    return cuda_check(cudaGetLastError(), "k_step_pair launch");
  }
}

// One state-to-state step (p in -> p out, no moments): paired or one-cell.
template <int Q, class S>
int launch_state_step(const lbm_plan* p, const lbm::StepArgs& m, cudaStream_t s) {
  if (pair_ok<S>(p, m)) return launch_pair<Q, S>(m, s);
  return launch_step<Q, S>(m, false, s);
}

template <int Q, class S>
int launch_step_padded(const lbm::StepArgs& a, cudaStream_t s) {
  const unsigned grid = grid_for(a.g.ncell);
  const bool faces = a.face[0].kind != lbm::kFaceNone || a.face[1].kind != lbm::kFaceNone;
  const bool force = a.force_mode != 0;
  if (faces) {
    if (force) lbm::k_step_padded<Q, S, true, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step_padded<Q, S, true, false><<<grid, lbm::kBlock, 0, s>>>(a);
  } else {
    if (force) lbm::k_step_padded<Q, S, false, true><<<grid, lbm::kBlock, 0, s>>>(a);
    else lbm::k_step_padded<Q, S, false, false><<<grid, lbm::kBlock, 0, s>>>(a);
  }
  return cuda_check(cudaGetLastError(), "k_step_padded launch");
}

// Collide the whole padded block into the workspace, then the padded step.
template <int Q, class S>
int run_padded(const lbm_plan* p, cudaStream_t s, lbm::StepArgs a, const void* f_in,
               void* f_out, char* ws) {
  (void)p;
  lbm::StepArgs m = a;
  m.rho = m.vel = m.prs = nullptr;  // halo moments stay the caller's
  m.f_in = f_in;
  m.pout = ws;
  int rc = launch_prepare<Q, S>(m, s);
  if (rc) return rc;
  a.pin = ws;
  a.f_in = f_in;
  a.f_out = f_out;
  return launch_step_padded<Q, S>(a, s);
}

template <int Q, class S>
int launch_step_moments_only(const lbm::StepArgs& a, cudaStream_t s) {
  launch_step_mode<Q, S, lbm::kOutMoments>(a, s);
  return cuda_check(cudaGetLastError(), "k_step launch");
}

// One-pass tiled step (lbm_tiled.cuh) for lbm_update and the first step of a
// rollout: 32-bit IO, rows of a multiple of 4 cells (16-byte copy groups),
// 16-byte aligned reference-layout buffers that do not overlap, an unpadded
// whole lattice.
template <class S>
bool tiled_ok(const lbm_plan* p, const lbm::StepArgs& a, const void* ws, bool aos_out) {
  if constexpr (sizeof(typename lbm::StoreT<S>::IO) != 4) {
    return false;
  } else {
    if (p->flags & LBM_PLAN_TWO_PASS) return false;
    if (p->g.n2 % 4 != 0 || p->g.rstride != p->g.n2 || a.face_inset != 0 || a.force_mode == 3)
      return false;
    const uintptr_t fi = reinterpret_cast<uintptr_t>(a.f_in);
    const uintptr_t fo = reinterpret_cast<uintptr_t>(a.f_out);
    if (fi % 16 != 0) return false;
    if (aos_out) {
      // f_out is written while other blocks still read f_in: no overlap
      const uintptr_t bytes = static_cast<uintptr_t>(p->g.ncell) * p->Q * 4;
      if (fo % 16 != 0 || (fo < fi + bytes && fi < fo + bytes)) return false;
    }
    return reinterpret_cast<uintptr_t>(ws) % 4 == 0;  // the status word
  }
}

// Runs the first step (one-pass tiled kernel, or prepare + a state step),
// the state steps and the final step; ws holds 1 or 2 state copies (with n > 1
// also the status word after them).
template <int Q, class S>
int run_steps(const lbm_plan* p, cudaStream_t s, lbm::StepArgs a, const void* f_in, void* f_out,
              int64_t n, char* ws) {
  const size_t sb = align256(state_bytes(p));
  char* A = ws;
  char* B = ws + sb;
  a.f_in = f_in;
  a.f_out = f_out;
  int rc;
  if constexpr (sizeof(typename lbm::StoreT<S>::IO) == 4) {
    if (n == 1 && tiled_ok<S>(p, a, ws, true)) {
      // the whole update in one pass; the workspace holds only the status word
      a.status = reinterpret_cast<int*>(ws);
      rc = cuda_check(cudaMemsetAsync(a.status, 0, sizeof(int), s), "cudaMemsetAsync");
      if (rc) return rc;
      return launch_tiled<Q, S, lbm::kOutAoS>(p, a, s);
    }
  }
  a.pout = A;
  lbm::StepArgs m = a;  // the first pass and intermediate steps write no moments
  m.rho = m.vel = m.prs = nullptr;
  const bool tiled = n > 1 && tiled_ok<S>(p, a, ws + 2 * sb, false);
  if (tiled) {
    m.status = reinterpret_cast<int*>(ws + 2 * sb);
    rc = cuda_check(cudaMemsetAsync(m.status, 0, sizeof(int), s), "cudaMemsetAsync");
    if (rc) return rc;
  }
  if (tiled) {
    // step 1 straight from the reference layout (p after one step into A)
    if constexpr (sizeof(typename lbm::StoreT<S>::IO) == 4)
      rc = launch_tiled<Q, S, lbm::kOutState>(p, m, s);
    --n;
  } else {
    rc = launch_prepare<Q, S>(m, s);
  }
  if (rc) return rc;
  for (int64_t i = 0; i + 1 < n; ++i) {
    m.pin = A;
    m.pout = B;
    rc = launch_state_step<Q, S>(p, m, s);
    if (rc) return rc;
    char* t = A;
    A = B;
    B = t;
  }
  a.pin = A;
  a.f_out = f_out;
  return launch_step<Q, S>(a, true, s);
}

// Rollout that also records the reference state after every `every`-th step
// (record r = after step (r + 1) every): recorded state steps write f and the
// moments into the history slots as they collide; the last step's outputs are
// copied into its slot when it is recorded.
template <int Q, class S>
int run_history(const lbm_plan* p, cudaStream_t s, lbm::StepArgs a, const void* f_in,
                void* f_out, int64_t n, int64_t every, const lbm_history* h, char* ws) {
  const size_t sb = align256(state_bytes(p));
  const size_t cells = p->g.ncell;
  const size_t fb = cells * p->Q * p->io, rb = cells * p->io, vb = cells * p->D * p->io;
  auto slot = [](void* base, size_t bytes, int64_t r) -> void* {
    return base == nullptr ? nullptr : static_cast<char*>(base) + static_cast<size_t>(r) * bytes;
  };
  char* A = ws;
  char* B = ws + sb;
  lbm::StepArgs m = a;
  m.rho = m.vel = m.prs = nullptr;
  m.f_in = f_in;
  m.pout = A;
  int rc = launch_prepare<Q, S>(m, s);
  if (rc) return rc;
  for (int64_t i = 1; i < n; ++i) {
    m.pin = A;
    m.pout = B;
    if (i % every == 0) {
      const int64_t r = i / every - 1;
      lbm::StepArgs rec = m;
      rec.f_out = slot(h->f, fb, r);
      rec.rho = slot(h->density, rb, r);
      rec.vel = slot(h->velocity, vb, r);
      rec.prs = slot(h->pressure, rb, r);
      launch_step_mode<Q, S, lbm::kOutRecord>(rec, s);
      rc = cuda_check(cudaGetLastError(), "k_step launch");
    } else {
      rc = launch_state_step<Q, S>(p, m, s);
    }
    if (rc) return rc;
    char* t = A;
    A = B;
    B = t;
  }
  const bool last = n % every == 0;
  const int64_t r = n / every - 1;
  a.pin = A;
  a.f_out = f_out;
  // the last step's moments go to the caller's buffers, or straight to the
  // history slot when the caller wants none
  if (last && a.rho == nullptr) a.rho = slot(h->density, rb, r);
  if (last && a.vel == nullptr) a.vel = slot(h->velocity, vb, r);
  if (last && a.prs == nullptr) a.prs = slot(h->pressure, rb, r);
  rc = launch_step<Q, S>(a, true, s);
  if (rc || !last) return rc;
  struct { void* dst; const void* src; size_t bytes; } copies[4] = {
      {slot(h->f, fb, r), f_out, fb},
      {slot(h->density, rb, r), a.rho, rb},
      {slot(h->velocity, vb, r), a.vel, vb},
      {slot(h->pressure, rb, r), a.prs, rb}};
  for (const auto& c : copies) {
    if (c.dst == nullptr || c.dst == c.src) continue;
    rc = cuda_check(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToDevice, s),
                    "cudaMemcpyAsync");
    if (rc) return rc;
  }
  return LBM_OK;
}

template <int Q>
int dispatch_s(const lbm_plan* p, cudaStream_t s, const lbm::StepArgs& a, const void* f_in,
               void* f_out, int64_t n, char* ws) {
  switch (p->storage) {
    case LBM_STORE_F32: return run_steps<Q, float>(p, s, a, f_in, f_out, n, ws);
    case LBM_STORE_F16: return run_steps<Q, __half>(p, s, a, f_in, f_out, n, ws);
    case LBM_STORE_BF16: return run_steps<Q, __nv_bfloat16>(p, s, a, f_in, f_out, n, ws);
    case LBM_STORE_F64: return run_steps<Q, double>(p, s, a, f_in, f_out, n, ws);
  }
  return fail(LBM_ERR_INVALID, "bad storage");
}

int do_steps(const lbm_plan* p, lbm_stream_t stream, const void* f_in, void* f_out, int64_t n,
             const lbm_step_args* args, const lbm_moments* out, void* workspace,
             size_t workspace_bytes, int nbuf) {
  if (p == nullptr) return fail(LBM_ERR_INVALID, "plan is NULL");
  if (f_in == nullptr || f_out == nullptr) return fail(LBM_ERR_INVALID, "f_in/f_out is NULL");
  if (n < 1) return fail(LBM_ERR_INVALID, "n_steps must be >= 1 (got %lld)", (long long)n);
  const size_t need = nbuf == 1 ? state_bytes(p) : 2 * align256(state_bytes(p)) + 256;
  if (workspace == nullptr || workspace_bytes < need)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", need,
                workspace_bytes);
  lbm::StepArgs a;
  int rc = build_args(p, args, out, &a);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  return p->Q == 19 ? dispatch_s<19>(p, s, a, f_in, f_out, n, ws)
                    : dispatch_s<9>(p, s, a, f_in, f_out, n, ws);
}

constexpr int kReduceBlocks = 148 * 4;

// ---------------------------------------------------------------------------
// Differentiated rollout: checkpointed forward + reverse sweep
// ---------------------------------------------------------------------------

struct AdjLayout {
  int64_t T = 0, K = 0, S = 0;  // steps, checkpoint interval, segments
  size_t sb = 0;                // bytes of one population copy
  size_t rho_bytes = 0, slot = 0;
  size_t A = 0, B = 0, ck = 0, hist = 0, mu0 = 0, mu1 = 0, dF = 0, part = 0, total = 0;
};

int adj_layout(const lbm_plan* p, int64_t T, int64_t K, AdjLayout* L) {
  if (T < 1) return fail(LBM_ERR_INVALID, "n_steps must be >= 1 (got %lld)", (long long)T);
  if (K <= 0) {
    K = 1;
    while (K * K < T) ++K;  // ceil(sqrt(T))
  }
  L->T = T;
  L->K = K;
  L->S = (T + K - 1) / K;
  L->sb = align256(state_bytes(p));
  L->rho_bytes = align256(static_cast<size_t>(p->g.ncell) * p->io);
  L->slot = L->rho_bytes + align256(static_cast<size_t>(p->g.ncell) * p->D * p->io);
  size_t o = 0;
  L->A = o; o += L->sb;
  L->B = o; o += L->sb;
  L->ck = o; o += static_cast<size_t>(L->S - 1) * L->sb;
  L->hist = o; o += static_cast<size_t>(K + 1) * L->slot;
  L->mu0 = o; o += L->sb;
  L->mu1 = o; o += L->sb;
  L->dF = o; o += align256(static_cast<size_t>(p->g.ncell) * p->D * sizeof(double));
  L->part = o; o += align256(sizeof(double) * 4 * kReduceBlocks);
  L->total = o;
  return LBM_OK;
}

int adj_check(const lbm_plan* p, const lbm_step_args* args) {
  if (p == nullptr || args == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  if (p->storage != LBM_STORE_F32 && p->storage != LBM_STORE_F64)
    return fail(LBM_ERR_UNSUPPORTED, "the differentiated rollout needs FP32 or FP64 storage");
  if (args->inlet.kind != LBM_BC_NONE || args->outlet.kind != LBM_BC_NONE)
    return fail(LBM_ERR_UNSUPPORTED,
                "the differentiated rollout supports walls and body forces, not face conditions");
  return LBM_OK;
}

template <int Q, class S>
int adj_forward(const lbm_plan* p, cudaStream_t s, lbm::StepArgs a, const void* f_in, void* f_out,
                const AdjLayout& L, char* ws) {
  char* AB[2] = {ws + L.A, ws + L.B};
  auto slot = [&](int64_t j) { return ws + L.ck + static_cast<size_t>(j - 1) * L.sb; };
  // Producer of p^m writes into checkpoint j = (m+1)/K when m+1 is a segment start.
  auto out_for = [&](int64_t m, char* cur) -> char* {
    if ((m + 1) % L.K == 0 && m + 1 < L.T) return slot((m + 1) / L.K);
    return cur == AB[0] ? AB[1] : AB[0];
  };
  lbm::StepArgs m = a;
  m.rho = m.vel = m.prs = nullptr;
  m.f_in = f_in;
  char* cur = out_for(0, nullptr);
  m.pout = cur;
  int rc = launch_prepare<Q, S>(m, s);
  if (rc) return rc;
  for (int64_t n = 1; n < L.T; ++n) {
    char* nxt = out_for(n, cur);
    m.pin = cur;
    m.pout = nxt;
    rc = launch_state_step<Q, S>(p, m, s);
    if (rc) return rc;
    cur = nxt;
  }
  a.pin = cur;
  a.f_out = f_out;
  return launch_step<Q, S>(a, true, s);
}

template <int Q, class S>
int adj_backward(const lbm_plan* p, cudaStream_t s, lbm::StepArgs a, const void* f_in,
                 const void* g_rho, const void* g_vel, const void* g_f, double* grad_force,
                 void* grad_f_in, const AdjLayout& L, char* ws) {
  using IO = typename lbm::StoreT<S>::IO;
  char* AB[2] = {ws + L.A, ws + L.B};
  char* MU[2] = {ws + L.mu0, ws + L.mu1};
  auto slot = [&](int64_t j) { return ws + L.ck + static_cast<size_t>(j - 1) * L.sb; };
  auto hist_rho = [&](int64_t j) { return ws + L.hist + static_cast<size_t>(j) * L.slot; };
  auto hist_vel = [&](int64_t j) { return hist_rho(j) + L.rho_bytes; };
  double* dF = reinterpret_cast<double*>(ws + L.dF);
  const unsigned grid = grid_for(p->g.ncell);

  lbm::AdjArgs q{};
  q.g = p->g;
  q.omega = a.omega;
  q.guo_c = a.guo_c;
  q.force_mode = a.force_mode;
  for (int d = 0; d < 3; ++d) q.force[d] = a.force[d];
  q.force_field = a.force_field;
  q.wall = a.wall;
  q.dF = grad_force != nullptr ? dF : nullptr;
  const bool force = a.force_mode != 0;

  lbm::StepArgs m = a;  // recompute steps: moments into the history, raw velocity
  m.prs = nullptr;
  m.mflags = lbm::kMomRawVelocity;
  m.f_in = f_in;
  int mu = 0;  // MU[mu] holds mu^{n+1}
  int rc = LBM_OK;
  for (int64_t sg = L.S - 1; sg >= 0; --sg) {
    const int64_t n0 = sg * L.K;
    const int64_t n1 = n0 + L.K < L.T ? n0 + L.K : L.T;
    // (rho^n, u^n) for n in [n0, n1): recompute from the segment's checkpoint
    char* cur = AB[0];
    m.rho = hist_rho(0);
    m.vel = hist_vel(0);
    m.pout = cur;
    if (sg == 0) {
      rc = launch_prepare<Q, S>(m, s);
    } else {
      m.pin = slot(sg);
      rc = launch_step<Q, S>(m, false, s);
    }
    if (rc) return rc;
    for (int64_t n = n0 + 1; n < n1; ++n) {
      char* nxt = cur == AB[0] ? AB[1] : AB[0];
      m.rho = hist_rho(n - n0);
      m.vel = hist_vel(n - n0);
      m.pin = cur;
      m.pout = nxt;
      rc = launch_step<Q, S>(m, false, s);
      if (rc) return rc;
      cur = nxt;
    }
    if (sg == L.S - 1) {
      // moments of f^T, then lambda^T from the output gradients
      m.rho = hist_rho(n1 - n0);
      m.vel = hist_vel(n1 - n0);
      m.pin = cur;
      rc = launch_step_moments_only<Q, S>(m, s);
      if (rc) return rc;
      q.rho = hist_rho(n1 - n0);
      q.vel = hist_vel(n1 - n0);
      q.g_rho = g_rho;
      q.g_vel = g_vel;
      q.g_f = g_f;
      q.mout = MU[mu];
      lbm::k_adj_init<Q, S><<<grid, lbm::kBlock, 0, s>>>(q);
      rc = cuda_check(cudaGetLastError(), "k_adj_init launch");
      if (rc) return rc;
    }
    for (int64_t n = n1 - 1; n >= n0; --n) {
      q.rho = hist_rho(n - n0);
      q.vel = hist_vel(n - n0);
      q.min = MU[mu];
      q.mout = MU[1 - mu];
      const bool aos = n == 0 && grad_f_in != nullptr;
      q.grad_f0 = grad_f_in;
      if (aos) {
        if (force) lbm::k_adj_step<Q, S, true, lbm::kAdjOutAoS><<<grid, lbm::kBlock, 0, s>>>(q);
        else lbm::k_adj_step<Q, S, false, lbm::kAdjOutAoS><<<grid, lbm::kBlock, 0, s>>>(q);
      } else {
        if (force) lbm::k_adj_step<Q, S, true, lbm::kAdjOutState><<<grid, lbm::kBlock, 0, s>>>(q);
        else lbm::k_adj_step<Q, S, false, lbm::kAdjOutState><<<grid, lbm::kBlock, 0, s>>>(q);
      }
      rc = cuda_check(cudaGetLastError(), "k_adj_step launch");
      if (rc) return rc;
      mu = 1 - mu;
    }
  }
  if (grad_force != nullptr) {
    if (a.force_mode == LBM_FORCE_UNIFORM) {
      double* part = reinterpret_cast<double*>(ws + L.part);
      if (p->D == 3)
        lbm::k_field_sum_part<3><<<kReduceBlocks, lbm::kReduceThreads, 0, s>>>(dF, p->g.ncell, part);
      else
        lbm::k_field_sum_part<2><<<kReduceBlocks, lbm::kReduceThreads, 0, s>>>(dF, p->g.ncell, part);
      lbm::k_field_sum_final<<<1, lbm::kReduceThreads, 0, s>>>(part, kReduceBlocks, p->D,
                                                              grad_force);
      rc = cuda_check(cudaGetLastError(), "k_field_sum launch");
    } else {
      rc = cuda_check(cudaMemcpyAsync(grad_force, dF,
                                      static_cast<size_t>(p->g.ncell) * p->D * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s),
                      "cudaMemcpyAsync");
    }
  }
  (void)sizeof(IO);
  return rc;
}

// ---------------------------------------------------------------------------
// Batched ensemble (host side)
// ---------------------------------------------------------------------------

// A contiguous range [t0, t1) of the tile list whose instances are stepped
// together; grid = blocks of the persistent launch for that range; pair = its
// state steps run the paired kernel (16-bit storage, even rows).
struct TileRange {
  uint32_t t0, t1;  // reference-layout tiles (prepare, one-cell steps, last step)
  uint32_t s0, s1;  // state-layout tiles (paired state steps)
  unsigned grid, sgrid;
  bool pair;        // state steps paired
  bool pad;         // ... with padded state rows
};

// Prepare pass over all tiles, then for each instance group its n - 1 state
// steps and its last step.  A group whose two population copies fit in L2
// stays there for all of its steps.
template <int Q, class S, int MODE, int SPEC>
void batched_launch(bool pair, bool pad, const lbm::StepArgs* args, const lbm::BatchTile* t,
                    uint32_t nt, unsigned grid, int which, cudaStream_t s) {
  if constexpr (MODE == lbm::kOutState && sizeof(S) == 2) {
    if (pair) {
      if (pad) lbm::k_batched_pair<Q, S, SPEC, true><<<grid, lbm::kBlock, 0, s>>>(args, t, nt, which);
      else lbm::k_batched_pair<Q, S, SPEC, false><<<grid, lbm::kBlock, 0, s>>>(args, t, nt, which);
      return;
    }
  }
  lbm::k_batched_step<Q, S, MODE, SPEC><<<grid, lbm::kBlock, 0, s>>>(args, t, nt, which);
}

// spec: 0 = per-tile run-time choice, else 1 + 2 FACES + FORCE shared by all members
template <int Q, class S, int MODE>
void batched_step(int spec, bool pair, bool pad, const lbm::StepArgs* args,
                  const lbm::BatchTile* t, uint32_t nt, unsigned grid, int which, cudaStream_t s) {
  switch (spec) {
    case 1: batched_launch<Q, S, MODE, 1>(pair, pad, args, t, nt, grid, which, s); break;
    case 2: batched_launch<Q, S, MODE, 2>(pair, pad, args, t, nt, grid, which, s); break;
    case 3: batched_launch<Q, S, MODE, 3>(pair, pad, args, t, nt, grid, which, s); break;
    case 4: batched_launch<Q, S, MODE, 4>(pair, pad, args, t, nt, grid, which, s); break;
    default: batched_launch<Q, S, MODE, 0>(pair, pad, args, t, nt, grid, which, s); break;
  }
}

template <int Q, class S>
int batched_run(const lbm::StepArgs* args, const lbm::BatchTile* tiles,
                const lbm::BatchTile* stiles, uint32_t ntiles, unsigned grid_all,
                const std::vector<TileRange>& groups, int64_t n, cudaStream_t s,
                cudaStream_t side, bool use_graph, int spec) {
  lbm::k_batched_prepare<Q, S><<<grid_all, lbm::kBlock, 0, s>>>(args, tiles, ntiles);
  int rc = cuda_check(cudaGetLastError(), "k_batched_prepare launch");
  if (rc) return rc;
  cudaStream_t ls = s;
  cudaGraph_t graph = nullptr;
  if (use_graph) {
    // The step sequence is recorded on the batch's own stream (capture only
    // records, nothing runs there) and replayed on the caller's stream, after
    // the work already queued on it.
    rc = cuda_check(cudaStreamBeginCapture(side, cudaStreamCaptureModeThreadLocal),
                    "cudaStreamBeginCapture");
    if (rc) return rc;
    ls = side;
  }
  for (const TileRange& r : groups) {
    const lbm::BatchTile* t = tiles + r.t0;
    const uint32_t nt = r.t1 - r.t0;
    for (int64_t k = 1; k < n; ++k) {
      if (r.pair)
        batched_step<Q, S, lbm::kOutState>(spec, true, r.pad, args, stiles + r.s0, r.s1 - r.s0,
                                           r.sgrid, static_cast<int>(k % 2), ls);
      else
        batched_step<Q, S, lbm::kOutState>(spec, false, false, args, t, nt, r.grid,
                                           static_cast<int>(k % 2), ls);
    }
    batched_step<Q, S, lbm::kOutAoS>(spec, false, false, args, t, nt, r.grid, 2, ls);
  }
  rc = cuda_check(cudaGetLastError(), "k_batched_step launch");
  if (use_graph) {
    const int rc2 = cuda_check(cudaStreamEndCapture(side, &graph), "cudaStreamEndCapture");
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (rc2) return rc2;
    cudaGraphExec_t exec = nullptr;
    rc = cuda_check(cudaGraphInstantiate(&exec, graph, 0), "cudaGraphInstantiate");
    cudaGraphDestroy(graph);
    if (rc) return rc;
    rc = cuda_check(cudaGraphLaunch(exec, s), "cudaGraphLaunch");
    cudaGraphExecDestroy(exec);  // released once the launched graph completes
  }
  return rc;
}

}  // namespace

constexpr int kTileOrders = 3;

struct lbm_batch {
  int n = 0, Q = 0, D = 0, storage = 0;
  std::vector<const lbm_plan*> plans;
  std::vector<lbm::Geo> sgeo;     // member geometry with its state-plane layout
  std::vector<size_t> state_off;  // instance i: two population copies at this offset
  size_t args_off = 0, tiles_off[kTileOrders] = {0, 0, 0}, stiles_off[kTileOrders] = {0, 0, 0};
  size_t total = 0;
  // [0] instance-major in member order, [1] round-robin across members,
  // [2] instance-major from the smallest member to the largest; tiles over the
  // reference layout (tiles) and over the state planes (stiles; they differ
  // for padded rows)
  std::vector<lbm::BatchTile> tiles[kTileOrders], stiles[kTileOrders];
  // members in the order of tile lists 0 and 2 (members whose state steps run
  // paired -- 16-bit storage -- first), with their first tile in each list
  std::vector<int> order[kTileOrders];
  std::vector<uint32_t> first_tile[kTileOrders], first_stile[kTileOrders];
  int npair = 0;  // number of those members: the first npair_even have even rows
  int npair_even = 0;
  cudaStream_t side = nullptr;
};

// Scratch of lbm_update_noalloc: one population copy, in the module's static
// device memory (every GPU that loads the library holds it until exit).  In
// host code this name is a host-side stand-in, not a device address; the
// device address comes from cudaGetSymbolAddress with the device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[LBM_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_noalloc_scratch in the current context, looked up on
// every call (cheap once the module is loaded there): an address kept from
// an earlier call could belong to a context that has since been reset or
// replaced.  The first lookup on a device loads the library's module there.
int noalloc_scratch(void** out) {
  void* p = nullptr;
  const int rc = cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
  if (rc) return rc;
  *out = p;
  return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_abi_version(void) { return LBM_ABI_VERSION; }

int lbm_last_error(char* buf, size_t len) {
  if (buf == nullptr || len == 0) return LBM_ERR_INVALID;
  std::snprintf(buf, len, "%s", g_last_error.c_str());
  return LBM_OK;
}

int lbm_plan_create(const lbm_desc* desc, lbm_plan** plan) {
  if (desc == nullptr || plan == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  *plan = nullptr;
  if (desc->lattice != LBM_D3Q19 && desc->lattice != LBM_D2Q9)
    return fail(LBM_ERR_INVALID, "Unknown lattice Q=%d. Supported: D3Q19 (19), D2Q9 (9).",
                desc->lattice);
  if (desc->storage < LBM_STORE_F32 || desc->storage > LBM_STORE_F64)
    return fail(LBM_ERR_INVALID, "unknown storage %d", desc->storage);
  if (!(desc->tau > 0.5) || !std::isfinite(desc->tau))
    return fail(LBM_ERR_INVALID, "tau must be > 0.5 (got %g). Increase viscosity.", desc->tau);
  constexpr uint32_t kKnownFlags = LBM_PLAN_SINGLE_CELLS | LBM_PLAN_PAIRED_CELLS |
                                   LBM_PLAN_TWO_PASS | LBM_PLAN_TEST_WAIT_TIMEOUT;
  if (desc->flags & ~kKnownFlags)
    return fail(LBM_ERR_INVALID, "unknown or reserved plan flags 0x%x",
                static_cast<unsigned>(desc->flags & ~kKnownFlags));
  lbm_plan* p = new lbm_plan();
  p->Q = desc->lattice;
  p->D = desc->lattice == LBM_D3Q19 ? 3 : 2;
  p->storage = desc->storage;
  p->tau = desc->tau;
  p->flags = desc->flags;
  int64_t dims[3];
  for (int d = 0; d < p->D; ++d) {
    if (desc->shape[d] < 1 || desc->shape[d] > (1 << 20)) {
      delete p;
      return fail(LBM_ERR_INVALID, "grid_shape[%d] = %lld out of range", d,
                  (long long)desc->shape[d]);
    }
    p->shape[d] = desc->shape[d];
  }
  if (p->D == 3) {
    dims[0] = p->shape[0]; dims[1] = p->shape[1]; dims[2] = p->shape[2];
  } else {
    dims[0] = 1; dims[1] = p->shape[0]; dims[2] = p->shape[1];
  }
  const int64_t ncell = dims[0] * dims[1] * dims[2];
  if (ncell * p->Q >= (int64_t(1) << 32)) {
    delete p;
    return fail(LBM_ERR_INVALID,
                "lattice of %lld cells is too large: Q x cells must stay below 2^32",
                (long long)ncell);
  }
  switch (p->storage) {
    case LBM_STORE_F32: p->elem = 4; p->io = 4; break;
    case LBM_STORE_F16:
    case LBM_STORE_BF16: p->elem = 2; p->io = 4; break;
    case LBM_STORE_F64: p->elem = 8; p->io = 8; break;
  }
  p->g.n0 = static_cast<uint32_t>(dims[0]);
  p->g.n1 = static_cast<uint32_t>(dims[1]);
  p->g.n2 = static_cast<uint32_t>(dims[2]);
  p->g.plane = static_cast<uint32_t>(dims[1] * dims[2]);
  p->g.ncell = static_cast<uint32_t>(ncell);
  p->g.div_n2 = make_fastdiv(p->g.n2);
  p->g.div_n1 = make_fastdiv(p->g.n1);
  p->g.rstride = p->g.n2;
  p->g.splane = p->g.plane;
  p->g.pstride = p->g.ncell;
  p->g.div_rstride = p->g.div_n2;
  if (!fastdiv_ok(p->g.div_n2, p->g.ncell) ||
      !fastdiv_ok(p->g.div_n1, static_cast<uint32_t>(dims[0] * dims[1]))) {
    delete p;
    return fail(LBM_ERR_INVALID, "internal: index division constants failed self-check");
  }
  *plan = p;
  return LBM_OK;
}

int lbm_plan_destroy(lbm_plan* plan) {
  delete plan;
  return LBM_OK;
}

int lbm_state_bytes(const lbm_plan* plan, size_t* bytes) {
  if (plan == nullptr || bytes == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  *bytes = state_bytes(plan);
  return LBM_OK;
}

int lbm_workspace_bytes(const lbm_plan* plan, size_t* bytes) {
  if (plan == nullptr || bytes == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  *bytes = 2 * align256(state_bytes(plan)) + 256;
  return LBM_OK;
}

int lbm_equilibrium(const lbm_plan* p, lbm_stream_t stream, const void* rho, const void* u,
                    void* f_out) {
  if (p == nullptr || f_out == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned grid = grid_for(p->g.ncell);
  if (p->io == 8) {
    if (p->Q == 19)
      lbm::k_equilibrium<19, double><<<grid, lbm::kBlock, 0, s>>>(
          p->g, static_cast<const double*>(rho), static_cast<const double*>(u),
          static_cast<double*>(f_out));
    else
      lbm::k_equilibrium<9, double><<<grid, lbm::kBlock, 0, s>>>(
          p->g, static_cast<const double*>(rho), static_cast<const double*>(u),
          static_cast<double*>(f_out));
  } else {
    if (p->Q == 19)
      lbm::k_equilibrium<19, float><<<grid, lbm::kBlock, 0, s>>>(
          p->g, static_cast<const float*>(rho), static_cast<const float*>(u),
          static_cast<float*>(f_out));
    else
      lbm::k_equilibrium<9, float><<<grid, lbm::kBlock, 0, s>>>(
          p->g, static_cast<const float*>(rho), static_cast<const float*>(u),
          static_cast<float*>(f_out));
  }
  return cuda_check(cudaGetLastError(), "k_equilibrium launch");
}

int lbm_update(const lbm_plan* plan, lbm_stream_t stream, const void* f_in, void* f_out,
               const lbm_step_args* args, const lbm_moments* out, void* workspace,
               size_t workspace_bytes) {
  return do_steps(plan, stream, f_in, f_out, 1, args, out, workspace, workspace_bytes, 1);
}

int lbm_rollout(const lbm_plan* plan, lbm_stream_t stream, const void* f_in, void* f_out,
                int64_t n_steps, const lbm_step_args* args, const lbm_moments* out,
                void* workspace, size_t workspace_bytes) {
  return do_steps(plan, stream, f_in, f_out, n_steps, args, out, workspace, workspace_bytes,
                  n_steps > 1 ? 2 : 1);
}

int lbm_rollout_history(const lbm_plan* p, lbm_stream_t stream, const void* f_in, void* f_out,
                        int64_t n_steps, int64_t every, const lbm_step_args* args,
                        const lbm_moments* out, const lbm_history* history, void* workspace,
                        size_t workspace_bytes) {
  if (p == nullptr) return fail(LBM_ERR_INVALID, "plan is NULL");
  if (f_in == nullptr || f_out == nullptr) return fail(LBM_ERR_INVALID, "f_in/f_out is NULL");
  if (history == nullptr) return fail(LBM_ERR_INVALID, "history is NULL");
  if (n_steps < 1) return fail(LBM_ERR_INVALID, "n_steps must be >= 1 (got %lld)", (long long)n_steps);
  if (every < 1) return fail(LBM_ERR_INVALID, "every must be >= 1 (got %lld)", (long long)every);
  const size_t need = 2 * align256(state_bytes(p)) + 256;
  if (workspace == nullptr || workspace_bytes < need)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", need,
                workspace_bytes);
  lbm::StepArgs a;
  int rc = build_args(p, args, out, &a);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  if (p->Q == 19) {
    switch (p->storage) {
      case LBM_STORE_F32: return run_history<19, float>(p, s, a, f_in, f_out, n_steps, every, history, ws);
      case LBM_STORE_F16: return run_history<19, __half>(p, s, a, f_in, f_out, n_steps, every, history, ws);
      case LBM_STORE_BF16: return run_history<19, __nv_bfloat16>(p, s, a, f_in, f_out, n_steps, every, history, ws);
      case LBM_STORE_F64: return run_history<19, double>(p, s, a, f_in, f_out, n_steps, every, history, ws);
    }
  } else {
    switch (p->storage) {
      case LBM_STORE_F32: return run_history<9, float>(p, s, a, f_in, f_out, n_steps, every, history, ws);
      case LBM_STORE_F16: return run_history<9, __half>(p, s, a, f_in, f_out, n_steps, every, history, ws);
      case LBM_STORE_BF16: return run_history<9, __nv_bfloat16>(p, s, a, f_in, f_out, n_steps, every, history, ws);
      case LBM_STORE_F64: return run_history<9, double>(p, s, a, f_in, f_out, n_steps, every, history, ws);
    }
  }
  return fail(LBM_ERR_INVALID, "bad storage");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Stepping the device state directly (the sharded runner)
// ---------------------------------------------------------------------------

namespace {

enum StateOp { kFromF, kStep, kToF };

template <int Q, class S>
int state_op(StateOp op, const lbm::StepArgs& a, cudaStream_t s) {
  if (op == kFromF) return launch_prepare<Q, S>(a, s);
  if (op == kStep) {
    launch_step_mode<Q, S, lbm::kOutState>(a, s);  // one cell per thread, any storage
    return cuda_check(cudaGetLastError(), "k_step launch");
  }
  return launch_step<Q, S>(a, true, s);
}

template <int Q>
int state_op_s(const lbm_plan* p, StateOp op, const lbm::StepArgs& a, cudaStream_t s) {
  switch (p->storage) {
    case LBM_STORE_F32: return state_op<Q, float>(op, a, s);
    case LBM_STORE_F16: return state_op<Q, __half>(op, a, s);
    case LBM_STORE_BF16: return state_op<Q, __nv_bfloat16>(op, a, s);
    case LBM_STORE_F64: return state_op<Q, double>(op, a, s);
  }
  return fail(LBM_ERR_INVALID, "bad storage");
}

int run_state_op(const lbm_plan* p, lbm_stream_t stream, StateOp op, const lbm::StepArgs& a) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return p->Q == 19 ? state_op_s<19>(p, op, a, s) : state_op_s<9>(p, op, a, s);
}

int state_args(const lbm_plan* p, const lbm_step_args* args, const lbm_moments* out,
               int64_t index_offset, lbm::StepArgs* a) {
  if (p == nullptr) return fail(LBM_ERR_INVALID, "plan is NULL");
  if (index_offset < 0) return fail(LBM_ERR_INVALID, "index_offset must be >= 0");
  const int rc = build_args(p, args, out, a);
  if (rc) return rc;
  // the rounding seed takes the index modulo 2^32, as for a whole lattice
  a->sr_offset = static_cast<uint32_t>(static_cast<uint64_t>(index_offset));
  return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_state_from_f(const lbm_plan* p, lbm_stream_t stream, const void* f_in, void* state_out,
                     const lbm_step_args* args, int64_t index_offset) {
  if (f_in == nullptr || state_out == nullptr)
    return fail(LBM_ERR_INVALID, "f_in/state_out is NULL");
  lbm::StepArgs a;
  int rc = state_args(p, args, nullptr, index_offset, &a);
  if (rc) return rc;
  a.f_in = f_in;
  a.pout = state_out;
  return run_state_op(p, stream, kFromF, a);
}

int lbm_state_step(const lbm_plan* p, lbm_stream_t stream, const void* state_in, void* state_out,
                   const lbm_step_args* args, int64_t first, int64_t count,
                   int64_t index_offset) {
  if (state_in == nullptr || state_out == nullptr)
    return fail(LBM_ERR_INVALID, "state_in/state_out is NULL");
  if (state_in == state_out) return fail(LBM_ERR_INVALID, "state_in must not be state_out");
  lbm::StepArgs a;
  int rc = state_args(p, args, nullptr, index_offset, &a);
  if (rc) return rc;
  if (first < 0 || count < 0 || first + count > p->shape[0])
    return fail(LBM_ERR_INVALID, "slices [%lld, %lld) outside axis 0 of extent %lld",
                (long long)first, (long long)(first + count), (long long)p->shape[0]);
  if (count == 0) return LBM_OK;
  const uint32_t slice = p->g.ncell / static_cast<uint32_t>(p->shape[0]);
  a.cell0 = static_cast<uint32_t>(first) * slice;
  a.cell_end = static_cast<uint32_t>(first + count) * slice;
  a.pin = state_in;
  a.pout = state_out;
  return run_state_op(p, stream, kStep, a);
}

int lbm_state_to_f(const lbm_plan* p, lbm_stream_t stream, const void* state_in, void* f_out,
                   const lbm_step_args* args, const lbm_moments* out) {
  if (state_in == nullptr || f_out == nullptr)
    return fail(LBM_ERR_INVALID, "state_in/f_out is NULL");
  lbm::StepArgs a;
  int rc = state_args(p, args, out, 0, &a);
  if (rc) return rc;
  a.pin = state_in;
  a.f_out = f_out;
  return run_state_op(p, stream, kToF, a);
}

}  // extern "C"

namespace {

size_t pipe_workspace(const lbm_plan* p) {
  const size_t n = p->g.ncell;
  return 2 * align256(state_bytes(p)) + 2 * align256(7 * n * p->io) + align256(3 * n * p->io);
}

// Single-phase pipe rollout: one fused launch per step (k_pipe_step: D3Q19
// pull step + the tracer of the same cell), tracer populations ping-ponged
// between two plane sets.
template <class S>
int run_pipe(const lbm_plan* p, cudaStream_t s, lbm::StepArgs a, const void* f_in, void* f_out,
             const void* t_in, void* t_out, int64_t n, double tau_tracer, void* tracer_out,
             char* ws) {
  using IO = typename lbm::StoreT<S>::IO;
  const size_t cells = p->g.ncell;
  const size_t sb = align256(state_bytes(p)), tb = align256(7 * cells * p->io);
  char* A = ws;
  char* B = ws + sb;
  char* T[2] = {ws + 2 * sb, ws + 2 * sb + tb};
  const unsigned grid = grid_for(p->g.ncell);
  lbm::TracerArgs t{};
  t.g = p->g;
  t.wall = a.wall;
  t.inv_tau = 1.0 / tau_tracer;
  t.f7_in = t_in;
  t.tout = T[0];
  lbm::k_tracer_prepare<IO><<<grid, lbm::kBlock, 0, s>>>(t);
  int rc = cuda_check(cudaGetLastError(), "k_tracer_prepare launch");
  if (rc) return rc;
  lbm::StepArgs m = a;
  m.rho = m.prs = m.vel = nullptr;
  m.f_in = f_in;
  m.pout = A;
  rc = launch_prepare<19, S>(m, s);
  if (rc) return rc;
  int cur = 0;
  for (int64_t i = 1; i < n; ++i) {
    m.pin = A;
    m.pout = B;
    t.tin = T[cur];
    t.tout = T[1 - cur];
    lbm::k_pipe_step<S, false><<<grid, lbm::kBlock, 0, s>>>(m, t);
    rc = cuda_check(cudaGetLastError(), "k_pipe_step launch");
    if (rc) return rc;
    cur = 1 - cur;
    std::swap(A, B);
  }
  a.pin = A;
  a.f_out = f_out;
  a.prs = nullptr;
  a.mflags &= ~lbm::kMomRawVelocity;
  t.tin = T[cur];
  t.tout = T[1 - cur];
  lbm::k_pipe_step<S, true><<<grid, lbm::kBlock, 0, s>>>(a, t);
  rc = cuda_check(cudaGetLastError(), "k_pipe_step launch");
  if (rc) return rc;
  cur = 1 - cur;
  t.tin = T[cur];
  t.f7_out = t_out;
  t.tracer_out = tracer_out;
  lbm::k_tracer_final<IO><<<grid, lbm::kBlock, 0, s>>>(t);
  return cuda_check(cudaGetLastError(), "k_tracer_final launch");
}

// Multiphase pipe step (G != 0): two passes per step over pre-collision
// population planes (lbm_multiphase.cuh); the workspace holds two population
// sets and the psi plane, inside the single-phase layout.
template <class R>
int run_pipe_mp(const lbm_plan* p, cudaStream_t s, const lbm::StepArgs& a,
                const lbm_pipe_args* pa, const void* f_in, void* f_out, const void* t_in,
                void* t_out, int64_t n, const lbm_moments* out, void* tracer_out, char* ws) {
  const size_t cells = p->g.ncell;
  const size_t sb = align256(state_bytes(p));
  char* A = ws;
  char* B = ws + sb;
  lbm::MPArgs m{};
  m.s = a;
  m.G = pa->G;
  m.rho0 = pa->rho_0;
  m.psi_wall = pa->rho_0 * (1.0 - std::exp(-pa->rho_wall / pa->rho_0));
  m.rho_gas = pa->rho_gas;
  m.drho = pa->rho_liquid - pa->rho_gas;
  m.psi = ws + 2 * sb;
  m.f_aos_in = f_in;
  const unsigned grid = grid_for(p->g.ncell);
  // step 1: psi of the reference f, then its collide into A
  lbm::k_mp_density<R, lbm::kMPFirst><<<grid, lbm::kBlock, 0, s>>>(m);
  int rc = cuda_check(cudaGetLastError(), "k_mp_density launch");
  if (rc) return rc;
  m.fout = A;
  lbm::k_mp_collide<R, true><<<grid, lbm::kBlock, 0, s>>>(m);
  rc = cuda_check(cudaGetLastError(), "k_mp_collide launch");
  if (rc) return rc;
  // steps 2..n: both passes pull from the post-collision planes
  for (int64_t i = 1; i < n; ++i) {
    m.fin = A;
    m.fout = B;
    lbm::k_mp_density<R, lbm::kMPStep><<<grid, lbm::kBlock, 0, s>>>(m);
    rc = cuda_check(cudaGetLastError(), "k_mp_density launch");
    if (rc) return rc;
    lbm::k_mp_collide<R, false><<<grid, lbm::kBlock, 0, s>>>(m);
    rc = cuda_check(cudaGetLastError(), "k_mp_collide launch");
    if (rc) return rc;
    std::swap(A, B);
  }
  m.fin = A;
  m.f_aos_out = f_out;
  m.rho_out = out != nullptr ? out->density : nullptr;
  m.vel_out = out != nullptr ? out->velocity : nullptr;
  m.tracer_out = tracer_out;
  lbm::k_mp_density<R, lbm::kMPLast><<<grid, lbm::kBlock, 0, s>>>(m);
  rc = cuda_check(cudaGetLastError(), "k_mp_density launch");
  if (rc) return rc;
  // tracer_f is not evolved in multiphase mode (lbm_pipe.py:858-860)
  return cuda_check(cudaMemcpyAsync(t_out, t_in, 7 * cells * sizeof(R), cudaMemcpyDeviceToDevice, s),
                    "tracer_f copy");
}

}  // namespace

extern "C" {

int lbm_pipe_workspace_bytes(const lbm_plan* plan, size_t* bytes) {
  if (plan == nullptr || bytes == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  *bytes = pipe_workspace(plan);
  return LBM_OK;
}

int lbm_pipe_rollout(const lbm_plan* p, lbm_stream_t stream, const void* f_in, void* f_out,
                     const void* tracer_f_in, void* tracer_f_out, int64_t n_steps,
                     const lbm_pipe_args* pa, const lbm_moments* out, void* tracer_out,
                     void* workspace, size_t workspace_bytes) {
  if (p == nullptr || pa == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  if (p->Q != 19) return fail(LBM_ERR_UNSUPPORTED, "the pipe node is D3Q19");
  if (p->storage != LBM_STORE_F32 && p->storage != LBM_STORE_F64)
    return fail(LBM_ERR_UNSUPPORTED, "the pipe node runs FP32 or FP64 storage");
  if (f_in == nullptr || f_out == nullptr || tracer_f_in == nullptr || tracer_f_out == nullptr)
    return fail(LBM_ERR_INVALID, "f / tracer_f is NULL");
  if (n_steps < 1) return fail(LBM_ERR_INVALID, "n_steps must be >= 1 (got %lld)", (long long)n_steps);
  if (!(pa->tau_tracer > 0.5)) return fail(LBM_ERR_INVALID, "tau_tracer must be > 0.5");
  if (pa->G != 0.0) {
    if (!(pa->rho_liquid > pa->rho_gas))
      return fail(LBM_ERR_INVALID, "rho_liquid must be > rho_gas (got %g <= %g)", pa->rho_liquid,
                  pa->rho_gas);
    if (!(pa->rho_gas > 0.0)) return fail(LBM_ERR_INVALID, "rho_gas must be > 0");
    if (!(pa->rho_0 > 0.0)) return fail(LBM_ERR_INVALID, "rho_0 must be > 0");
  }
  if (pa->propeller != nullptr &&
      (pa->propeller_x < 0 || pa->propeller_x >= static_cast<int32_t>(p->g.n0)))
    return fail(LBM_ERR_INVALID, "propeller_x %d outside [0, %u)", pa->propeller_x, p->g.n0);
  const size_t need = pipe_workspace(p);
  if (workspace == nullptr || workspace_bytes < need)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", need,
                workspace_bytes);
  lbm_step_args sa{};
  sa.force_mode = LBM_FORCE_NONE;
  sa.wall = pa->wall;
  lbm::StepArgs a;
  int rc = build_args(p, &sa, out, &a);
  if (rc) return rc;
  a.force_mode = 3;
  a.force[0] = pa->propeller != nullptr ? pa->propeller_force : 0.0;
  a.force[1] = 0.0;
  a.force[2] = pa->gravity;
  a.prop_x = pa->propeller != nullptr ? static_cast<uint32_t>(pa->propeller_x) : 0xffffffffu;
  a.prop_mask = pa->propeller;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  if (pa->G != 0.0) {
    if (p->storage == LBM_STORE_F32)
      return run_pipe_mp<float>(p, s, a, pa, f_in, f_out, tracer_f_in, tracer_f_out, n_steps, out,
                                tracer_out, ws);
    return run_pipe_mp<double>(p, s, a, pa, f_in, f_out, tracer_f_in, tracer_f_out, n_steps, out,
                               tracer_out, ws);
  }
  if (p->storage == LBM_STORE_F32)
    return run_pipe<float>(p, s, a, f_in, f_out, tracer_f_in, tracer_f_out, n_steps,
                           pa->tau_tracer, tracer_out, ws);
  return run_pipe<double>(p, s, a, f_in, f_out, tracer_f_in, tracer_f_out, n_steps,
                          pa->tau_tracer, tracer_out, ws);
}

int lbm_update_padded(const lbm_plan* p, lbm_stream_t stream, const void* f_pad,
                      void* f_out_pad, const lbm_step_args* args, const lbm_moments* out,
                      void* workspace, size_t workspace_bytes) {
  if (p == nullptr) return fail(LBM_ERR_INVALID, "plan is NULL");
  if (f_pad == nullptr || f_out_pad == nullptr) return fail(LBM_ERR_INVALID, "f is NULL");
  for (int d = 0; d < p->D; ++d)
    if (p->shape[d] < 3)
      return fail(LBM_ERR_INVALID,
                  "padded extent %lld along axis %d: one halo cell per side needs >= 3",
                  (long long)p->shape[d], d);
  const size_t need = state_bytes(p);
  if (workspace == nullptr || workspace_bytes < need)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", need,
                workspace_bytes);
  lbm::StepArgs a;
  int rc = build_args(p, args, out, &a);
  if (rc) return rc;
  a.face_inset = 1;
  if (a.face[1].kind == lbm::kFaceZeroGrad && p->shape[a.face[1].ref_axis] < 5)
    return fail(LBM_ERR_INVALID,
                "zero-gradient face needs >= 3 interior cells along axis %d",
                a.face[1].ref_axis);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  if (p->Q == 19) {
    switch (p->storage) {
      case LBM_STORE_F32: return run_padded<19, float>(p, s, a, f_pad, f_out_pad, ws);
      case LBM_STORE_F16: return run_padded<19, __half>(p, s, a, f_pad, f_out_pad, ws);
      case LBM_STORE_BF16: return run_padded<19, __nv_bfloat16>(p, s, a, f_pad, f_out_pad, ws);
      case LBM_STORE_F64: return run_padded<19, double>(p, s, a, f_pad, f_out_pad, ws);
    }
  } else {
    switch (p->storage) {
      case LBM_STORE_F32: return run_padded<9, float>(p, s, a, f_pad, f_out_pad, ws);
      case LBM_STORE_F16: return run_padded<9, __half>(p, s, a, f_pad, f_out_pad, ws);
      case LBM_STORE_BF16: return run_padded<9, __nv_bfloat16>(p, s, a, f_pad, f_out_pad, ws);
      case LBM_STORE_F64: return run_padded<9, double>(p, s, a, f_pad, f_out_pad, ws);
    }
  }
  return fail(LBM_ERR_INVALID, "bad storage");
}

int lbm_update_noalloc(const lbm_plan* plan, lbm_stream_t stream, const void* f_in,
                       void* f_out, const lbm_step_args* args, const lbm_moments* out) {
  if (plan == nullptr) return fail(LBM_ERR_INVALID, "plan is NULL");
  const size_t need = state_bytes(plan);
  if (need > LBM_NOALLOC_SCRATCH_BYTES)
    return fail(LBM_ERR_WORKSPACE,
                "lbm_update_noalloc: this lattice needs %zu bytes of scratch, more than the "
                "%u-byte static array; use lbm_update with a workspace",
                need, static_cast<unsigned>(LBM_NOALLOC_SCRATCH_BYTES));
  void* ws = nullptr;
  const int rc = noalloc_scratch(&ws);
  if (rc) return rc;
  return do_steps(plan, stream, f_in, f_out, 1, args, out, ws, LBM_NOALLOC_SCRATCH_BYTES, 1);
}

int lbm_adjoint_workspace_bytes(const lbm_plan* plan, int64_t n_steps, int64_t checkpoint_every,
                                size_t* bytes) {
  if (plan == nullptr || bytes == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  AdjLayout L;
  const int rc = adj_layout(plan, n_steps, checkpoint_every, &L);
  if (rc) return rc;
  *bytes = L.total;
  return LBM_OK;
}

int lbm_rollout_forward(const lbm_plan* p, lbm_stream_t stream, const void* f_in, void* f_out,
                        int64_t n_steps, int64_t checkpoint_every, const lbm_step_args* args,
                        const lbm_moments* out, void* workspace, size_t workspace_bytes) {
  int rc = adj_check(p, args);
  if (rc) return rc;
  if (f_in == nullptr || f_out == nullptr) return fail(LBM_ERR_INVALID, "f_in/f_out is NULL");
  AdjLayout L;
  rc = adj_layout(p, n_steps, checkpoint_every, &L);
  if (rc) return rc;
  if (workspace == nullptr || workspace_bytes < L.total)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", L.total,
                workspace_bytes);
  lbm::StepArgs a;
  rc = build_args(p, args, out, &a);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  if (p->storage == LBM_STORE_F64)
    return p->Q == 19 ? adj_forward<19, double>(p, s, a, f_in, f_out, L, ws)
                      : adj_forward<9, double>(p, s, a, f_in, f_out, L, ws);
  return p->Q == 19 ? adj_forward<19, float>(p, s, a, f_in, f_out, L, ws)
                    : adj_forward<9, float>(p, s, a, f_in, f_out, L, ws);
}

int lbm_rollout_backward(const lbm_plan* p, lbm_stream_t stream, const void* f_in,
                         int64_t n_steps, int64_t checkpoint_every, const lbm_step_args* args,
                         const void* grad_density, const void* grad_velocity, const void* grad_f,
                         double* grad_force, void* grad_f_in, void* workspace,
                         size_t workspace_bytes) {
  int rc = adj_check(p, args);
  if (rc) return rc;
  if (f_in == nullptr) return fail(LBM_ERR_INVALID, "f_in is NULL");
  AdjLayout L;
  rc = adj_layout(p, n_steps, checkpoint_every, &L);
  if (rc) return rc;
  if (workspace == nullptr || workspace_bytes < L.total)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", L.total,
                workspace_bytes);
  lbm::StepArgs a;
  rc = build_args(p, args, nullptr, &a);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  if (p->storage == LBM_STORE_F64)
    return p->Q == 19 ? adj_backward<19, double>(p, s, a, f_in, grad_density, grad_velocity,
                                                 grad_f, grad_force, grad_f_in, L, ws)
                      : adj_backward<9, double>(p, s, a, f_in, grad_density, grad_velocity,
                                                grad_f, grad_force, grad_f_in, L, ws);
  return p->Q == 19 ? adj_backward<19, float>(p, s, a, f_in, grad_density, grad_velocity, grad_f,
                                              grad_force, grad_f_in, L, ws)
                    : adj_backward<9, float>(p, s, a, f_in, grad_density, grad_velocity, grad_f,
                                             grad_force, grad_f_in, L, ws);
}

int lbm_batch_create(const lbm_plan* const* plans, int32_t n, lbm_batch** out) {
  if (plans == nullptr || out == nullptr || n < 1) return fail(LBM_ERR_INVALID, "bad arguments");
  *out = nullptr;
  lbm_batch* b = new lbm_batch();
  b->n = n;
  b->Q = plans[0] ? plans[0]->Q : 0;
  b->D = plans[0] ? plans[0]->D : 0;
  b->storage = plans[0] ? plans[0]->storage : 0;
  size_t o = 0;
  b->args_off = o;
  o += align256(sizeof(lbm::StepArgs) * lbm::kBatchArgs * static_cast<size_t>(n));
  const bool half = b->storage == LBM_STORE_F16 || b->storage == LBM_STORE_BF16;
  auto pairable = [&](int i) { return half && !(plans[i]->flags & LBM_PLAN_SINGLE_CELLS); };
  std::vector<std::vector<lbm::BatchTile>> per(n), sper(n);
  size_t ntiles = 0, nstiles = 0;
  for (int i = 0; i < n; ++i) {
    const lbm_plan* p = plans[i];
    if (p == nullptr || p->Q != b->Q || p->storage != b->storage) {
      delete b;
      return fail(LBM_ERR_INVALID, "instance %d: plans must share lattice and storage", i);
    }
    b->plans.push_back(p);
    // A paired member with odd rows keeps its state rows padded to n2 + 1.
    lbm::Geo g = p->g;
    if (pairable(i) && g.n2 % 2 == 1) {
      const uint64_t rs = uint64_t(g.n2) + 1;
      const uint64_t ps = uint64_t(g.n0) * g.n1 * rs;
      g.rstride = static_cast<uint32_t>(rs);
      g.splane = static_cast<uint32_t>(uint64_t(g.n1) * rs);
      g.div_rstride = make_fastdiv(g.rstride);
      if (ps * p->Q >= (uint64_t(1) << 32) || !fastdiv_ok(g.div_rstride, static_cast<uint32_t>(ps))) {
        delete b;
        return fail(LBM_ERR_INVALID, "instance %d: padded rows exceed 32-bit indexing", i);
      }
      g.pstride = static_cast<uint32_t>(ps);
    }
    b->sgeo.push_back(g);
    for (uint32_t c = 0; c < g.ncell; c += lbm::kBatchTile)
      per[i].push_back(lbm::BatchTile{static_cast<uint32_t>(i), c});
    for (uint32_t c = 0; c < g.pstride; c += lbm::kBatchTile)
      sper[i].push_back(lbm::BatchTile{static_cast<uint32_t>(i), c});
    ntiles += per[i].size();
    nstiles += sper[i].size();
  }
  if (nstiles >= (size_t(1) << 31)) {
    delete b;
    return fail(LBM_ERR_INVALID, "ensemble too large");
  }
  std::vector<int> by_member(n), by_size(n);
  for (int i = 0; i < n; ++i) by_member[i] = by_size[i] = i;
  std::stable_sort(by_size.begin(), by_size.end(),
                   [&](int x, int y) { return plans[x]->g.ncell < plans[y]->g.ncell; });
  // classes: paired with even rows, paired with padded rows, one cell
  auto cls = [&](int i) { return !pairable(i) ? 2 : (plans[i]->g.n2 % 2 == 0 ? 0 : 1); };
  for (auto* v : {&by_member, &by_size})
    std::stable_sort(v->begin(), v->end(), [&](int x, int y) { return cls(x) < cls(y); });
  for (int i = 0; i < n; ++i) {
    b->npair += cls(i) < 2 ? 1 : 0;
    b->npair_even += cls(i) == 0 ? 1 : 0;
  }
  for (int k : {0, 2}) {
    for (int j = 0; j < n; ++j) {
      const int i = k == 0 ? by_member[j] : by_size[j];
      b->order[k].push_back(i);
      b->first_tile[k].push_back(static_cast<uint32_t>(b->tiles[k].size()));
      b->first_stile[k].push_back(static_cast<uint32_t>(b->stiles[k].size()));
      b->tiles[k].insert(b->tiles[k].end(), per[i].begin(), per[i].end());
      b->stiles[k].insert(b->stiles[k].end(), sper[i].begin(), sper[i].end());
    }
  }
  for (size_t r = 0;; ++r) {  // round-robin across instances (one-cell steps only)
    bool any = false;
    for (int i = 0; i < n; ++i)
      if (r < per[i].size()) { b->tiles[1].push_back(per[i][r]); any = true; }
    if (!any) break;
  }
  for (int k = 0; k < kTileOrders; ++k) {
    b->tiles_off[k] = o;
    o += align256(sizeof(lbm::BatchTile) * ntiles);
    b->stiles_off[k] = o;
    o += align256(sizeof(lbm::BatchTile) * (k == 1 ? 1 : nstiles));
  }
  for (int i = 0; i < n; ++i) {
    b->state_off.push_back(o);
    const size_t sb = static_cast<size_t>(b->Q) * b->sgeo[i].pstride * plans[i]->elem;
    o += 2 * align256(sb);
  }
  b->total = o;
  if (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess) b->side = nullptr;
  *out = b;
  return LBM_OK;
}

int lbm_batch_destroy(lbm_batch* b) {
  if (b != nullptr && b->side != nullptr) cudaStreamDestroy(b->side);
  delete b;
  return LBM_OK;
}

int lbm_batch_workspace_bytes(const lbm_batch* b, size_t* bytes) {
  if (b == nullptr || bytes == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  *bytes = b->total;
  return LBM_OK;
}

int lbm_batch_rollout(const lbm_batch* b, lbm_stream_t stream, const void* const* f_in,
                      void* const* f_out, int64_t n_steps, const lbm_step_args* args,
                      const lbm_moments* out, const lbm_batch_config* cfg, void* workspace,
                      size_t workspace_bytes) {
  if (b == nullptr || f_in == nullptr || f_out == nullptr || args == nullptr)
    return fail(LBM_ERR_INVALID, "NULL argument");
  if (n_steps < 1) return fail(LBM_ERR_INVALID, "n_steps must be >= 1 (got %lld)", (long long)n_steps);
  if (workspace == nullptr || workspace_bytes < b->total)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", b->total,
                workspace_bytes);
  lbm_batch_config c{0, 0, 0, 0};
  if (cfg != nullptr) c = *cfg;
  if (c.tile_order < 0 || c.tile_order >= kTileOrders || c.blocks_per_sm < 0 || c.group_mib < 0)
    return fail(LBM_ERR_INVALID, "bad batch config");
  if (c.group_mib > 0 && c.tile_order == 1)
    return fail(LBM_ERR_INVALID, "instance groups need an instance-major tile order (0 or 2)");
  if (c.use_graph && b->side == nullptr)
    return fail(LBM_ERR_UNSUPPORTED, "no capture stream for CUDA-graph replay");
  char* ws = static_cast<char*>(workspace);
  std::vector<lbm::StepArgs> host(static_cast<size_t>(lbm::kBatchArgs) * b->n);
  for (int i = 0; i < b->n; ++i) {
    const lbm_plan* p = b->plans[i];
    if (f_in[i] == nullptr || f_out[i] == nullptr)
      return fail(LBM_ERR_INVALID, "instance %d: f_in/f_out is NULL", i);
    lbm::StepArgs a;
    int rc = build_args(p, &args[i], out != nullptr ? &out[i] : nullptr, &a);
    if (rc) return rc;
    a.g = b->sgeo[i];  // the member's state-plane layout (padded rows or not)
    char* A = ws + b->state_off[i];
    char* B = A + align256(static_cast<size_t>(b->Q) * a.g.pstride * p->elem);
    lbm::StepArgs m = a;
    m.rho = m.vel = m.prs = nullptr;
    m.f_in = f_in[i];
    lbm::StepArgs* h = &host[static_cast<size_t>(lbm::kBatchArgs) * i];
    h[0] = m;
    h[0].pin = B;
    h[0].pout = A;
    h[1] = m;
    h[1].pin = A;
    h[1].pout = B;
    h[2] = a;  // last step: p^{n-1} is in A when n is odd, else in B
    h[2].pin = n_steps % 2 == 1 ? A : B;
    h[2].f_out = f_out[i];
  }
  // One face / force specialisation shared by every member: compile-time kernel.
  int spec = -1;
  for (int i = 0; i < b->n; ++i) {
    const lbm::StepArgs& h = host[static_cast<size_t>(lbm::kBatchArgs) * i];
    const bool faces = h.face[0].kind != lbm::kFaceNone || h.face[1].kind != lbm::kFaceNone;
    const int si = 1 + 2 * (faces ? 1 : 0) + (h.force_mode != 0 ? 1 : 0);
    spec = spec < 0 || spec == si ? si : 0;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  lbm::StepArgs* dargs = reinterpret_cast<lbm::StepArgs*>(ws + b->args_off);
  lbm::BatchTile* dtiles = reinterpret_cast<lbm::BatchTile*>(ws + b->tiles_off[c.tile_order]);
  lbm::BatchTile* dstiles = reinterpret_cast<lbm::BatchTile*>(ws + b->stiles_off[c.tile_order]);
  const auto& tl = b->tiles[c.tile_order];
  const auto& stl = b->stiles[c.tile_order];
  int rc = cuda_check(cudaMemcpyAsync(dargs, host.data(), host.size() * sizeof(lbm::StepArgs),
                                      cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
  if (rc) return rc;
  rc = cuda_check(cudaMemcpyAsync(dtiles, tl.data(), tl.size() * sizeof(lbm::BatchTile),
                                  cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
  if (rc) return rc;
  if (!stl.empty()) {
    rc = cuda_check(cudaMemcpyAsync(dstiles, stl.data(), stl.size() * sizeof(lbm::BatchTile),
                                    cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    if (rc) return rc;
  }
  const uint32_t ntiles = static_cast<uint32_t>(tl.size());
  unsigned cap = 0;  // persistent grid size, 0 = one block per tile
  if (c.blocks_per_sm > 0) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cap = static_cast<unsigned>(c.blocks_per_sm) * static_cast<unsigned>(sms);
  }
  auto grid_for_tiles = [cap](uint32_t nt) { return cap > 0 && cap < nt ? cap : nt; };
  // Instance groups: consecutive members of the tile order whose two
  // population copies together stay within group_mib (a member larger than
  // that is a group of its own); 0 = all members in every launch.
  // Members whose state steps run paired come first in tile orders 0 and 2;
  // members with even rows read their wall mask two bytes at a time, so it
  // must be 2-byte aligned (else nothing runs paired).
  int npair = c.tile_order == 1 ? 0 : b->npair;
  for (int j = 0; j < npair; ++j) {
    const int i = b->order[c.tile_order][j];
    if (b->sgeo[i].rstride == b->sgeo[i].n2 && reinterpret_cast<uintptr_t>(args[i].wall) % 2 != 0)
      npair = 0;
  }
  const size_t jeven = npair > 0 ? static_cast<size_t>(b->npair_even) : 0u;
  std::vector<TileRange> groups;
  const auto& ord = b->order[c.tile_order];
  const auto& ft = b->first_tile[c.tile_order];
  const auto& fs = b->first_stile[c.tile_order];
  const uint32_t nstiles = static_cast<uint32_t>(stl.size());
  // member j of the order -> its first reference / state tile (end = totals)
  auto tile_at = [&](size_t j) { return j < ord.size() ? ft[j] : ntiles; };
  auto stile_at = [&](size_t j) { return j < ord.size() ? fs[j] : nstiles; };
  const size_t jsplit = static_cast<size_t>(npair);
  // members [0, jeven) paired, [jeven, jsplit) paired with padded rows, the rest one cell
  auto add_range = [&](size_t j0, size_t j1) {
    const uint32_t t0 = tile_at(j0), t1 = tile_at(j1);
    if (t1 <= t0) return;
    const bool pair = j0 < jsplit, pad = pair && j0 >= jeven;
    const uint32_t s0 = pair ? stile_at(j0) : 0u, s1 = pair ? stile_at(j1) : 0u;
    groups.push_back(TileRange{t0, t1, s0, s1, grid_for_tiles(t1 - t0),
                               grid_for_tiles(s1 - s0), pair, pad});
  };
  if (c.tile_order == 1) {
    groups.push_back(TileRange{0, ntiles, 0, 0, grid_for_tiles(ntiles), 0, false, false});
  } else if (c.group_mib == 0) {
    add_range(0, jeven);
    add_range(jeven, jsplit);
    add_range(jsplit, ord.size());
  } else {
    const size_t budget = static_cast<size_t>(c.group_mib) << 20;
    size_t used = 0, j0 = 0;
    for (size_t j = 0; j < ord.size(); ++j) {
      const size_t need =
          2 * align256(static_cast<size_t>(b->Q) * b->sgeo[ord[j]].pstride * b->plans[ord[j]]->elem);
      if (j > 0 && (used + need > budget || j == jeven || j == jsplit)) {
        add_range(j0, j);
        j0 = j;
        used = 0;
      }
      used += need;
    }
    add_range(j0, ord.size());
  }
  const unsigned grid_all = grid_for_tiles(ntiles);
  const bool g = c.use_graph != 0;
#define LBM_BATCH_RUN(QQ, SS) \
  batched_run<QQ, SS>(dargs, dtiles, dstiles, ntiles, grid_all, groups, n_steps, s, b->side, \
                      g, spec)
  switch (b->storage) {
    case LBM_STORE_F32: return b->Q == 19 ? LBM_BATCH_RUN(19, float) : LBM_BATCH_RUN(9, float);
    case LBM_STORE_F16: return b->Q == 19 ? LBM_BATCH_RUN(19, __half) : LBM_BATCH_RUN(9, __half);
    case LBM_STORE_BF16:
      return b->Q == 19 ? LBM_BATCH_RUN(19, __nv_bfloat16) : LBM_BATCH_RUN(9, __nv_bfloat16);
    case LBM_STORE_F64: return b->Q == 19 ? LBM_BATCH_RUN(19, double) : LBM_BATCH_RUN(9, double);
  }
#undef LBM_BATCH_RUN
  return fail(LBM_ERR_INVALID, "bad storage");
}

int lbm_reduce_workspace_bytes(const lbm_plan* plan, size_t* bytes) {
  if (plan == nullptr || bytes == nullptr) return fail(LBM_ERR_INVALID, "NULL argument");
  *bytes = sizeof(double) * 4 * kReduceBlocks;
  return LBM_OK;
}

int lbm_mass_momentum(const lbm_plan* p, lbm_stream_t stream, const void* f, double* out_dev,
                      void* workspace, size_t workspace_bytes) {
  if (p == nullptr || f == nullptr || out_dev == nullptr)
    return fail(LBM_ERR_INVALID, "NULL argument");
  const size_t need = sizeof(double) * 4 * kReduceBlocks;
  if (workspace == nullptr || workspace_bytes < need)
    return fail(LBM_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", need,
                workspace_bytes);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(workspace);
  const double nc = static_cast<double>(p->g.ncell);
  if (p->io == 8) {
    if (p->Q == 19) {
      lbm::k_mass_momentum_part<19, double><<<kReduceBlocks, lbm::kReduceThreads, 0, s>>>(
          p->g, static_cast<const double*>(f), part);
      lbm::k_mass_momentum_final<19><<<1, lbm::kReduceThreads, 0, s>>>(part, kReduceBlocks, nc, out_dev);
    } else {
      lbm::k_mass_momentum_part<9, double><<<kReduceBlocks, lbm::kReduceThreads, 0, s>>>(
          p->g, static_cast<const double*>(f), part);
      lbm::k_mass_momentum_final<9><<<1, lbm::kReduceThreads, 0, s>>>(part, kReduceBlocks, nc, out_dev);
    }
  } else {
    if (p->Q == 19) {
      lbm::k_mass_momentum_part<19, float><<<kReduceBlocks, lbm::kReduceThreads, 0, s>>>(
          p->g, static_cast<const float*>(f), part);
      lbm::k_mass_momentum_final<19><<<1, lbm::kReduceThreads, 0, s>>>(part, kReduceBlocks, nc, out_dev);
    } else {
      lbm::k_mass_momentum_part<9, float><<<kReduceBlocks, lbm::kReduceThreads, 0, s>>>(
          p->g, static_cast<const float*>(f), part);
      lbm::k_mass_momentum_final<9><<<1, lbm::kReduceThreads, 0, s>>>(part, kReduceBlocks, nc, out_dev);
    }
  }
  return cuda_check(cudaGetLastError(), "k_mass_momentum launch");
}

int lbm_pack_f32(lbm_stream_t stream, const lbm_pack_field* fields, int32_t n_fields,
                 float* out, int64_t out_count) {
  if (n_fields < 0) return fail(LBM_ERR_INVALID, "n_fields must be >= 0 (got %d)", n_fields);
  if (n_fields > 0 && fields == nullptr) return fail(LBM_ERR_INVALID, "fields is NULL");
  int64_t total = 0;
  for (int32_t i = 0; i < n_fields; ++i) {
    const lbm_pack_field& f = fields[i];
    if (f.count < 0) return fail(LBM_ERR_INVALID, "field %d: count %lld < 0", i, (long long)f.count);
    if (f.offset < 0) return fail(LBM_ERR_INVALID, "field %d: offset %lld < 0", i, (long long)f.offset);
    if (f.count > 0 && f.data == nullptr) return fail(LBM_ERR_INVALID, "field %d: data is NULL", i);
    if (f.dtype < LBM_DTYPE_F32 || f.dtype > LBM_DTYPE_I64)
      return fail(LBM_ERR_INVALID, "field %d: unknown dtype %d", i, f.dtype);
    if (f.offset + f.count > out_count)
      return fail(LBM_ERR_INVALID, "field %d: elements [%lld, %lld) outside the payload of %lld",
                  i, (long long)f.offset, (long long)(f.offset + f.count), (long long)out_count);
    total += f.count;
  }
  if (total > 0 && out == nullptr) return fail(LBM_ERR_INVALID, "out is NULL");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  for (int32_t first = 0; first < n_fields; first += lbm::kPackMaxFields) {
    const int32_t nb = std::min<int32_t>(lbm::kPackMaxFields, n_fields - first);
    lbm::PackBatch b{};
    int64_t most = 0;
    for (int32_t j = 0; j < nb; ++j) {
      const lbm_pack_field& f = fields[first + j];
      b.src[j] = f.data;
      b.count[j] = f.count;
      b.offset[j] = f.offset;
      b.type[j] = f.dtype;
      most = std::max(most, f.count);
    }
    if (most == 0) continue;
    const int64_t want = (most + 4 * lbm::kPackThreads - 1) / (4 * lbm::kPackThreads);
    const unsigned gx = static_cast<unsigned>(std::min<int64_t>(want, 148 * 8));
    lbm::k_pack_f32<<<dim3(gx, nb), lbm::kPackThreads, 0, s>>>(b, out);
    const int rc = cuda_check(cudaGetLastError(), "k_pack_f32 launch");
    if (rc) return rc;
  }
  return LBM_OK;
}

}  // extern "C"
