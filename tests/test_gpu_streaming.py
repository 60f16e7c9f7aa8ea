"""Streaming frames with device-resident state: the ``lbm_pack_f32`` gather
(one launch for all device fields, one transfer) gives the same frame bytes as
the reference's encoder on the host (fixtures from ``api/binary_encoder.py``),
for every dtype the states hold; more fields than one launch takes; a frame of
a running LBMNode."""

import numpy as np
import pytest
import torch

from maddening_b200.streaming import BinaryStateEncoder, decode_frame
from tests.golden.make_golden import FRAME_SUBSCRIPTIONS, frame_states

pytestmark = pytest.mark.gpu


def _to_device(state):
    """Arrays to CUDA tensors; Python scalars stay on the host."""
    return {n: {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray)
                    else v) for k, v in fields.items()} for n, fields in state.items()}


@pytest.mark.parametrize("sub", list(FRAME_SUBSCRIPTIONS))
@pytest.mark.parametrize("sname", ["rods", "lattice"])
def test_device_frames_match_reference(golden, sname, sub):
    state = _to_device(frame_states()[sname])
    enc = BinaryStateEncoder(state, fields=FRAME_SUBSCRIPTIONS[sub])
    frame = enc.encode(0.125 * len(sname), state)
    assert frame == golden[f"frame|{sname}|{sub}|bytes"].tobytes()
    assert enc.encode(0.125 * len(sname), state) == frame  # buffers reused


def test_all_dtypes_and_many_fields():
    g = torch.Generator(device="cuda").manual_seed(3)
    fields = {}
    for i in range(45):  # more than one launch's 32 fields
        n = 1 + 997 * i
        base = torch.randn(n, generator=g, device="cuda", dtype=torch.float64) * 10 ** (i % 5)
        dtype = (torch.float32, torch.float16, torch.bfloat16, torch.float64, torch.uint8,
                 torch.int32, torch.int64, torch.bool)[i % 8]
        if dtype in (torch.uint8, torch.bool):
            v = (base.abs() * 7).to(torch.uint8) if dtype is torch.uint8 else base > 0
        else:
            v = base.to(dtype)
        fields[f"x{i:02d}"] = v
    state = {"node": fields}
    enc = BinaryStateEncoder(state)
    payload = enc.encode_device(state)
    expect = torch.cat([fields[k].flatten().to(torch.float64).to(torch.float32)
                        if fields[k].dtype == torch.float64 else fields[k].flatten().float()
                        for k in sorted(fields)])
    assert torch.equal(payload, expect)
    t, values = decode_frame(enc.encode(2.0, state), enc.schema())
    assert t == 2.0 and np.array_equal(values, expect.cpu().numpy())


def test_frame_of_a_running_node():
    from maddening_b200 import LBMNode
    node = LBMNode("vessel", 1.0, grid_shape=(32, 24, 20), viscosity=0.1)
    st = node.run(node.initial_state(), {"body_force": np.array([1e-5, 0.0, 0.0])}, 20)
    state = {"vessel": st, "heart": {"pressure": 12.0}}
    enc = BinaryStateEncoder(state, fields={"vessel": ["density", "velocity"],
                                            "heart": ["pressure"]})
    t, values = decode_frame(enc.encode(20.0, state), enc.schema())
    host = {"vessel": {k: st[k].cpu().numpy() for k in ("density", "velocity")},
            "heart": {"pressure": 12.0}}
    ref = BinaryStateEncoder(host, fields={"vessel": ["density", "velocity"],
                                           "heart": ["pressure"]})
    assert enc.encode(20.0, state) == ref.encode(20.0, host)
    assert values.size == 32 * 24 * 20 * 4 + 1
