"""The C ABI driven from plain C: a C program (no Python, no torch in its
process) creates a D3Q19 FP32 plan, reads a seeded state and wall mask, runs
``lbm_update`` with a velocity inlet and a zero-gradient outlet (the one-pass
kernel) and writes f_bc and the moments; ``LBMNode.update`` on the same inputs
gives the same bytes.  The program links ``liblbm_b200.so`` and the CUDA
runtime the way a C or C++ caller of the reference-facing boundary would."""

import os
import subprocess
import tempfile

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "maddening_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SHAPE = (16, 12, 20)

PROG = r"""
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime_api.h>
#include "lbm_b200.h"

#define LBM(x) do { int rc_ = (x); if (rc_ != LBM_OK) { char m_[512]; \
  lbm_last_error(m_, sizeof m_); fprintf(stderr, "%s: %d %s\n", #x, rc_, m_); return 1; } } while (0)
#define CU(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
  fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_)); return 1; } } while (0)

static int read_all(const char* path, void* buf, size_t n) {
  FILE* fp = fopen(path, "rb");
  if (!fp) return 1;
  size_t got = fread(buf, 1, n, fp);
  fclose(fp);
  return got != n;
}

static int write_all(const char* path, const void* buf, size_t n) {
  FILE* fp = fopen(path, "wb");
  if (!fp) return 1;
  size_t put = fwrite(buf, 1, n, fp);
  fclose(fp);
  return put != n;
}

int main(int argc, char** argv) {
  if (argc != 4) return 2;  /* f_in, wall, output prefix */
  const size_t n0 = N0, n1 = N1, n2 = N2, ncell = n0 * n1 * n2, nf = ncell * 19;
  lbm_desc d = {0};
  d.lattice = LBM_D3Q19;
  d.storage = LBM_STORE_F32;
  d.shape[0] = n0; d.shape[1] = n1; d.shape[2] = n2;
  d.tau = TAU;
  lbm_plan* plan = NULL;
  LBM(lbm_plan_create(&d, &plan));

  float* f = (float*)malloc(nf * 4);
  unsigned char* wall = (unsigned char*)malloc(ncell);
  float* out = (float*)malloc(nf * 4);
  if (!f || !wall || !out) return 3;
  if (read_all(argv[1], f, nf * 4) || read_all(argv[2], wall, ncell)) return 4;

  void *df, *dout, *dwall, *drho, *dvel, *dprs, *dws;
  size_t ws = 0;
  LBM(lbm_workspace_bytes(plan, &ws));
  CU(cudaMalloc(&df, nf * 4));
  CU(cudaMalloc(&dout, nf * 4));
  CU(cudaMalloc(&dwall, ncell));
  CU(cudaMalloc(&drho, ncell * 4));
  CU(cudaMalloc(&dvel, ncell * 12));
  CU(cudaMalloc(&dprs, ncell * 4));
  CU(cudaMalloc(&dws, ws));
  CU(cudaMemcpy(df, f, nf * 4, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dwall, wall, ncell, cudaMemcpyHostToDevice));

  lbm_step_args a = {0};
  a.force_mode = LBM_FORCE_NONE;
  a.wall = (const uint8_t*)dwall;
  a.inlet.kind = LBM_BC_VELOCITY;
  a.inlet.face = LBM_FACE_X_MIN;
  a.inlet.value[0] = UIN;
  a.outlet.kind = LBM_BC_ZERO_GRADIENT;
  a.outlet.face = LBM_FACE_X_MAX;
  lbm_moments m = {0};
  m.density = drho;
  m.velocity = dvel;
  m.pressure = dprs;
  LBM(lbm_update(plan, NULL, df, dout, &a, &m, dws, ws));
  CU(cudaDeviceSynchronize());

  char path[4096];
  CU(cudaMemcpy(out, dout, nf * 4, cudaMemcpyDeviceToHost));
  snprintf(path, sizeof path, "%s_f.bin", argv[3]);
  if (write_all(path, out, nf * 4)) return 5;
  CU(cudaMemcpy(out, drho, ncell * 4, cudaMemcpyDeviceToHost));
  snprintf(path, sizeof path, "%s_rho.bin", argv[3]);
  if (write_all(path, out, ncell * 4)) return 5;
  CU(cudaMemcpy(out, dvel, ncell * 12, cudaMemcpyDeviceToHost));
  snprintf(path, sizeof path, "%s_vel.bin", argv[3]);
  if (write_all(path, out, ncell * 12)) return 5;

  LBM(lbm_plan_destroy(plan));
  cudaFree(df); cudaFree(dout); cudaFree(dwall); cudaFree(drho); cudaFree(dvel);
  cudaFree(dprs); cudaFree(dws);
  free(f); free(wall); free(out);
  printf("ok\n");
  return 0;
}
"""


def test_c_program_update_equals_node_update():
    from maddening_b200 import LBMNode
    tau, u_in = 0.8, 0.05
    rng = np.random.default_rng(11)
    wall = rng.random(SHAPE) < 0.1
    node = LBMNode("c", 1.0, grid_shape=SHAPE, viscosity=(tau - 0.5) / 3.0, wall_mask=wall,
                   outlet_condition="zero_gradient")
    assert abs(node.tau - tau) < 1e-12
    f = (node.lattice.w * (1 + 1e-2 * rng.standard_normal(SHAPE + (19,)))).astype(np.float32)
    bi = {"inlet_velocity": np.array([u_in, 0.0, 0.0], dtype=np.float32)}
    st = node.initial_state()
    st["f"] = torch.as_tensor(f, device="cuda")
    ref = node.update(st, bi, 1.0)

    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "drive.c"), os.path.join(d, "drive")
        defs = {"N0": SHAPE[0], "N1": SHAPE[1], "N2": SHAPE[2], "TAU": repr(float(node.tau)),
                "UIN": repr(float(np.float32(u_in)))}
        with open(src, "w") as fh:
            fh.write("".join(f"#define {k} {v}\n" for k, v in defs.items()) + PROG)
        subprocess.run(["gcc", "-O1", "-I", os.path.join(ROOT, "include"),
                        "-I", os.path.join(CUDA, "include"), src, "-o", exe,
                        "-L", PKG, "-llbm_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
                        f"-Wl,-rpath,{PKG}:{os.path.join(CUDA, 'lib64')}"], check=True)
        f.tofile(os.path.join(d, "f.bin"))
        wall.astype(np.uint8).tofile(os.path.join(d, "wall.bin"))
        run = subprocess.run([exe, os.path.join(d, "f.bin"), os.path.join(d, "wall.bin"),
                              os.path.join(d, "out")], capture_output=True, text=True, timeout=120)
        assert run.returncode == 0 and run.stdout.strip() == "ok", run.stderr
        got_f = np.fromfile(os.path.join(d, "out_f.bin"), dtype=np.float32).reshape(SHAPE + (19,))
        got_rho = np.fromfile(os.path.join(d, "out_rho.bin"), dtype=np.float32).reshape(SHAPE)
        got_vel = np.fromfile(os.path.join(d, "out_vel.bin"), dtype=np.float32).reshape(SHAPE + (3,))
    assert np.array_equal(got_f, ref["f"].cpu().numpy())
    assert np.array_equal(got_rho, ref["density"].cpu().numpy())
    assert np.array_equal(got_vel, ref["velocity"].cpu().numpy())
