"""Binary state frames for streaming simulation state.

Drop-in for MADDENING's ``src/maddening/api/binary_encoder.py``: a fixed
schema is built once from an example state ``{node: {field: value}}`` (nodes
and fields in sorted order, optionally restricted to a subscription), and
every frame is ``[8 B sim_time, float64][total_floats x 4 B float32 payload]``
with the values in schema order -- the same schema dict, frame bytes and
``decode_frame`` as the reference.

Device-resident fields (CUDA tensors: the node states of this package) are
converted to float32 and gathered into one device payload by a single
``lbm_pack_f32`` launch, then copied to pinned host memory in one transfer;
the state itself (e.g. a (grid, 19) population array) never crosses to the
host unless it is subscribed.  Host values (NumPy arrays, Python scalars, CPU
tensors) are written on the host.  A frame is assembled in one pinned host
buffer; ``encode`` copies it once into the returned bytes, ``encode_view``
hands out a view of the buffer itself, and ``encode_device`` returns the
payload as a device tensor for consumers on the GPU.

Compression (``"zstd"``, ``"zstd+xor"``) follows the reference and needs the
``zstandard`` package; without it the constructor raises ``ImportError``.
"""

from __future__ import annotations

import ctypes as C
import struct
from typing import Any

import numpy as np
import torch

from . import _lib

try:
    import zstandard as _zstd
    _HAS_ZSTD = True
except ImportError:  # not installed on this image
    _zstd = None
    _HAS_ZSTD = False

VALID_COMPRESSIONS = {"none", "zstd", "zstd+xor"}

_DTYPE_CODE = {torch.float32: 0, torch.float16: 1, torch.bfloat16: 2, torch.float64: 3,
               torch.uint8: 4, torch.bool: 4, torch.int32: 5, torch.int64: 6}


class lbm_pack_field(C.Structure):
    _fields_ = [("data", C.c_void_p), ("count", C.c_int64), ("offset", C.c_int64),
                ("dtype", C.c_int32)]


def _lib_pack():
    h = _lib.lib()
    if not getattr(h, "_pack_sigs", False):
        h.lbm_pack_f32.argtypes = [C.c_void_p, C.POINTER(lbm_pack_field), C.c_int32, C.c_void_p,
                                   C.c_int64]
        h.lbm_pack_f32.restype = C.c_int
        h._pack_sigs = True
    return h


def _count(val) -> tuple[tuple, int]:
    if hasattr(val, "shape"):
        shape = tuple(int(d) for d in val.shape)
        return shape, (max(1, int(np.prod(shape))) if shape else 1)
    return (), 1


class BinaryStateEncoder:
    """Fixed-schema float32 frames of a state dict (binary_encoder.py:40-229).

    Parameters follow the reference: ``state`` is an example
    ``{node_name: {field_name: array_or_scalar}}``; ``fields`` an optional
    ``{node_name: [field, ...]}`` subscription (unknown nodes and fields are
    ignored, an empty dict selects nothing); ``compression`` one of
    ``"none"``, ``"zstd"``, ``"zstd+xor"``; ``zstd_level`` 1-22.
    """

    def __init__(self, state: dict[str, dict[str, Any]], fields: dict[str, list[str]] | None = None,
                 *, compression: str = "none", zstd_level: int = 3):
        if compression not in VALID_COMPRESSIONS:
            raise ValueError(f"compression must be one of {VALID_COMPRESSIONS!r}, "
                             f"got {compression!r}")
        if compression != "none" and not _HAS_ZSTD:
            raise ImportError(f"compression={compression!r} requires the 'zstandard' "
                              "package. Install with: pip install maddening[compression]")
        self._compression = compression
        self._zstd_level = zstd_level
        self._cctx = _zstd.ZstdCompressor(level=zstd_level) if compression != "none" else None
        self._prev_payload: bytes | None = None
        self._subscription = fields
        self._fields: list[tuple[str, str, tuple, int]] = []
        self._total_floats = 0
        for node in sorted(state.keys()):
            if fields is not None and node not in fields:
                continue
            allowed = None if fields is None else set(fields[node])
            for field in sorted(state[node].keys()):
                if allowed is not None and field not in allowed:
                    continue
                shape, n = _count(state[node][field])
                self._fields.append((node, field, shape, n))
                self._total_floats += n
        self._buf_size = 8 + self._total_floats * 4
        self._dev_payload: dict[torch.device, torch.Tensor] = {}
        self._frame: torch.Tensor | None = None

    # -- schema ---------------------------------------------------------------
    def schema(self) -> dict:
        """JSON-serialisable layout of the payload (binary_encoder.py:127-149)."""
        out, offset = [], 0
        for node, field, shape, n in self._fields:
            out.append({"node": node, "field": field, "shape": list(shape), "offset": offset,
                        "count": n})
            offset += n
        return {"type": "schema", "fields": out, "total_floats": self._total_floats,
                "frame_bytes": self._buf_size, "compression": self._compression}

    @property
    def total_floats(self) -> int:
        return self._total_floats

    @property
    def frame_bytes(self) -> int:
        """Uncompressed frame size in bytes (8 + 4 total_floats)."""
        return self._buf_size

    @property
    def subscription(self):
        return self._subscription

    @property
    def compression(self) -> str:
        return self._compression

    # -- packing --------------------------------------------------------------
    def _split(self, state):
        """(device fields by device, host fields) of the schema, with offsets."""
        dev, host, offset = {}, [], 0
        for node, field, _shape, n in self._fields:
            val = state[node][field]
            if isinstance(val, torch.Tensor) and val.is_cuda:
                if val.numel() != n:
                    raise ValueError(f"{node}.{field}: {val.numel()} elements, schema has {n}")
                dev.setdefault(val.device, []).append((val, offset, n))
            else:
                host.append((val, offset, n))
            offset += n
        return dev, host

    def _pack_on(self, device, items) -> torch.Tensor:
        """Pack the device fields into the payload buffer of ``device``."""
        buf = self._dev_payload.get(device)
        if buf is None:
            buf = torch.empty(max(1, self._total_floats), dtype=torch.float32, device=device)
            self._dev_payload[device] = buf
        # keep: contiguous / converted copies stay referenced until the launch
        # is queued (the caching allocator orders any reuse on this stream)
        keep, descs = [], []
        for val, offset, n in items:
            t = val.contiguous()
            if t.dtype not in _DTYPE_CODE:
                t = t.to(torch.float32)
            keep.append(t)
            descs.append(lbm_pack_field(t.data_ptr(), n, offset, _DTYPE_CODE[t.dtype]))
        arr = (lbm_pack_field * len(descs))(*descs)
        stream = torch.cuda.current_stream(device).cuda_stream
        _lib.check(_lib_pack().lbm_pack_f32(stream, arr, len(descs), buf.data_ptr(),
                                            self._total_floats))
        return buf

    def encode_device(self, state: dict) -> torch.Tensor:
        """The float32 payload as a device tensor (all subscribed fields must
        live on one CUDA device).  It is the encoder's own buffer: valid until
        the next encode call on that device."""
        dev, host = self._split(state)
        if host or len(dev) != 1:
            raise ValueError("encode_device needs every subscribed field on one CUDA device")
        (device, items), = dev.items()
        return self._pack_on(device, items)[: self._total_floats]

    def _fill_frame(self, sim_time: float, state) -> np.ndarray:
        """The uncompressed frame in the encoder's own (pinned) host buffer:
        ``[8 B sim_time][payload]``, as a uint8 array over that buffer."""
        if self._frame is None:
            self._frame = torch.empty(self._buf_size, dtype=torch.uint8,
                                      pin_memory=torch.cuda.is_available())
        frame = self._frame.numpy()
        struct.pack_into("d", frame, 0, sim_time)
        if self._total_floats == 0:
            return frame
        payload = self._frame[8:].view(torch.float32)
        dev, host = self._split(state)
        for device, items in dev.items():
            buf = self._pack_on(device, items)
            if len(dev) == 1:  # one transfer; host fields are written over it below
                payload.copy_(buf[: self._total_floats], non_blocking=True)
            else:
                for _val, offset, n in items:
                    payload[offset: offset + n].copy_(buf[offset: offset + n], non_blocking=True)
            torch.cuda.current_stream(device).synchronize()
        out = payload.numpy()
        for val, offset, n in host:
            if isinstance(val, torch.Tensor):
                val = val.detach().numpy()
            if hasattr(val, "flatten"):
                out[offset: offset + n] = np.asarray(val.flatten(), dtype=np.float32)
            else:
                out[offset] = np.float32(float(val))
        return frame

    def encode_view(self, sim_time: float, state: dict) -> memoryview:
        """The uncompressed frame without a host-side copy: a view of the
        encoder's pinned frame buffer, valid until the next encode call (for
        senders that take a buffer, e.g. a WebSocket ``send_bytes``)."""
        if self._compression != "none":
            raise ValueError("encode_view gives uncompressed frames; use encode")
        return memoryview(self._fill_frame(sim_time, state))

    def encode(self, sim_time: float, state: dict) -> bytes:
        """``[8 B sim_time][payload]``, the payload compressed when asked
        (binary_encoder.py:151-205).  Uncompressed, the frame is assembled in
        the pinned buffer and copied once into the returned bytes."""
        frame = self._fill_frame(sim_time, state)
        if self._compression == "none":
            return frame.tobytes()
        payload = frame[8:].tobytes()
        if self._compression == "zstd":
            wire = self._cctx.compress(payload)
        else:  # zstd+xor: XOR against the previous payload, then compress
            if self._prev_payload is None or len(self._prev_payload) != len(payload):
                xored = payload
            else:
                a = np.frombuffer(payload, dtype=np.uint8)
                b = np.frombuffer(self._prev_payload, dtype=np.uint8)
                xored = (a ^ b).tobytes()
            wire = self._cctx.compress(xored)
            self._prev_payload = payload
        return struct.pack("d", sim_time) + wire


def decode_frame(frame: bytes, schema: dict) -> tuple[float, np.ndarray]:
    """Inverse of ``encode`` (binary_encoder.py:232-258): ``(sim_time, values)``."""
    sim_time = struct.unpack_from("d", frame, 0)[0]
    body = frame[8:]
    comp = schema.get("compression", "none")
    if comp == "none":
        raw = body
    elif comp == "zstd":
        if not _HAS_ZSTD:
            raise ImportError("zstandard not installed; cannot decode zstd-compressed frame")
        raw = _zstd.ZstdDecompressor().decompress(body)
    elif comp == "zstd+xor":
        raise NotImplementedError("zstd+xor decoding is stateful; the caller must maintain the "
                                  "previous payload and XOR after decompressing")
    else:
        raise ValueError(f"unknown compression {comp!r}")
    return sim_time, np.frombuffer(raw, dtype=np.float32)


__all__ = ["BinaryStateEncoder", "decode_frame", "VALID_COMPRESSIONS"]
