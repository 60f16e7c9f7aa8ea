"""The uneven-ensemble configuration (64 D3Q19 lattices, extents 32-160 per
axis, tau 0.55-1.5, z walls, body force g_x 1e-7-1e-5, 500 steps from rest)
with FP16 offset storage, batched, against the same ensemble with FP64
storage: every member's velocity within 1e-3 relative L2."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = a.double(), b.double()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_fp16_ensemble_members_within_1e3_of_fp64():
    from maddening_b200.batched import LBMEnsemble, uneven_ensemble
    n16, bis = uneven_ensemble(64, seed=0, storage="f16")
    n64, _ = uneven_ensemble(64, seed=0, storage="f64")
    o16 = LBMEnsemble(n16).run([n.initial_state() for n in n16], bis, 500)
    o64 = LBMEnsemble(n64).run([n.initial_state() for n in n64], bis, 500)
    errs = [_rel(a["velocity"], b["velocity"]) for a, b in zip(o16, o64)]
    worst = int(np.argmax(errs))
    assert max(errs) <= 1e-3, (worst, errs[worst], n16[worst].params, bis[worst])
