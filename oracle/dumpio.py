"""Reader for the binary dumps written by oracle/ref_dump.c.

TEST INFRASTRUCTURE ONLY (used by tests/golden/make_golden.py to turn dumps of
the reference into fixtures).

Format: b"CM3DDUMP", then records of
    char name[32]; int32 kind (1 = float64, 2 = int32); int64 count; payload,
terminated by b"ENDDUMP!".
"""
from __future__ import annotations

import struct

import numpy as np


def read_dump(path: str) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    with open(path, "rb") as fh:
        buf = fh.read()
    if buf[:8] != b"CM3DDUMP":
        raise ValueError(f"{path}: not a CM3D dump")
    pos = 8
    while pos < len(buf):
        if buf[pos:pos + 8] == b"ENDDUMP!":
            return out
        name = buf[pos:pos + 32].split(b"\0", 1)[0].decode()
        kind, count = struct.unpack_from("<iq", buf, pos + 32)
        pos += 32 + 4 + 8
        dt = np.float64 if kind == 1 else np.int32
        nbytes = count * (8 if kind == 1 else 4)
        out[name] = np.frombuffer(buf, dtype=dt, count=count, offset=pos).copy()
        pos += nbytes
    raise ValueError(f"{path}: truncated dump (no end marker)")
