"""Streaming frames (``maddening_b200/streaming.py``) on the host: the frames
and schemas the reference's own ``api/binary_encoder.py`` writes for the
fixture states (``tests/golden/make_golden.py``), and the behaviour its tests
check (tests/api/test_binary_encoder.py)."""

import json
import struct

import numpy as np
import pytest

from maddening_b200.streaming import _HAS_ZSTD, BinaryStateEncoder, decode_frame
from tests.golden.make_golden import FRAME_SUBSCRIPTIONS, frame_states


@pytest.mark.parametrize("sub", list(FRAME_SUBSCRIPTIONS))
@pytest.mark.parametrize("sname", ["rods", "lattice"])
def test_frames_match_reference(golden, sname, sub):
    state = frame_states()[sname]
    enc = BinaryStateEncoder(state, fields=FRAME_SUBSCRIPTIONS[sub])
    key = f"frame|{sname}|{sub}"
    assert enc.schema() == json.loads(str(golden[key + "|schema"]))
    frame = enc.encode(0.125 * len(sname), state)
    assert frame == golden[key + "|bytes"].tobytes()


@pytest.fixture
def sample_state():
    return frame_states()["rods"]


def test_schema_and_offsets(sample_state):
    schema = BinaryStateEncoder(sample_state).schema()
    assert schema["type"] == "schema"
    assert schema["total_floats"] == 23
    assert schema["frame_bytes"] == 8 + 23 * 4
    assert [f["node"] for f in schema["fields"]] == sorted(f["node"] for f in schema["fields"])
    offset = 0
    for f in schema["fields"]:
        assert f["offset"] == offset
        offset += f["count"]
    assert offset == schema["total_floats"]


def test_round_trip_and_frames(sample_state):
    enc = BinaryStateEncoder(sample_state)
    for i in range(5):
        frame = enc.encode(i * 0.01, sample_state)
        assert len(frame) == enc.frame_bytes
        t, values = decode_frame(frame, enc.schema())
        assert t == pytest.approx(i * 0.01, abs=1e-12)
        assert values.dtype == np.float32 and len(values) == 23
    fields = {(f["node"], f["field"]): f for f in enc.schema()["fields"]}
    assert values[fields[("ball", "velocity")]["offset"]] == np.float32(-3.2)
    rod = fields[("heat_rod", "temperature")]
    assert np.all(values[rod["offset"]: rod["offset"] + rod["count"]] == 20.0)


def test_scalars_and_empty():
    enc = BinaryStateEncoder({"a": {"x": 1.0, "y": 2}})
    assert enc.total_floats == 2 and enc.frame_bytes == 16
    assert decode_frame(enc.encode(0.5, {"a": {"x": 1.0, "y": 2}}), enc.schema())[1].tolist() == [1.0, 2.0]
    empty = BinaryStateEncoder({})
    assert empty.total_floats == 0 and empty.frame_bytes == 8
    frame = empty.encode(1.5, {})
    assert len(frame) == 8 and struct.unpack("d", frame)[0] == 1.5


def test_subscriptions(sample_state):
    enc = BinaryStateEncoder(sample_state, fields={"ball": ["position"]})
    assert enc.total_floats == 1 and enc.schema()["fields"][0]["field"] == "position"
    assert len(enc.encode(0.0, sample_state)) == 12
    enc = BinaryStateEncoder(sample_state, fields={"ball": ["velocity"], "heat_rod": ["temperature"]})
    assert enc.total_floats == 21
    assert BinaryStateEncoder(sample_state, fields={"ball": ["position", "nope"]}).total_floats == 1
    assert BinaryStateEncoder(sample_state, fields={"ball": ["position"], "x": ["y"]}).total_floats == 1
    assert BinaryStateEncoder(sample_state, fields={}).frame_bytes == 8
    sub = {"ball": ["position"]}
    assert BinaryStateEncoder(sample_state, fields=sub).subscription is sub
    assert BinaryStateEncoder(sample_state).subscription is None


def test_subset_reduces_a_lattice_frame():
    n = 32 ** 3
    big = {"lbm": {"velocity": np.zeros((n, 3), np.float32),
                   **{f"f{i}": np.zeros(n, np.float32) for i in range(19)}}}
    full, sub = BinaryStateEncoder(big), BinaryStateEncoder(big, fields={"lbm": ["velocity"]})
    assert 1.0 - sub.frame_bytes / full.frame_bytes > 0.80


def test_compression_modes(sample_state):
    with pytest.raises(ValueError, match="compression"):
        BinaryStateEncoder(sample_state, compression="lzma")
    assert BinaryStateEncoder(sample_state).compression == "none"
    if not _HAS_ZSTD:
        with pytest.raises(ImportError, match="zstandard"):
            BinaryStateEncoder(sample_state, compression="zstd")
    with pytest.raises(NotImplementedError):
        decode_frame(b"\0" * 8, {"compression": "zstd+xor"})


def test_encode_view_is_the_frame(sample_state):
    enc = BinaryStateEncoder(sample_state)
    view = enc.encode_view(1.25, sample_state)
    assert bytes(view) == enc.encode(1.25, sample_state)
    assert len(view) == enc.frame_bytes
