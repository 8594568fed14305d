"""Test infrastructure: reader for the operand dumps written by the reference
build's link-time hooks (oracle/ref_hooks.c)."""

from __future__ import annotations

import glob
import os
import struct

import numpy as np


def read_dump(path: str) -> dict:
    """Return {'tag', 'dt', 'time', 'recompute', 'vectors': [(origin, array)]}.

    Each array is (nz+2, ny+2, nx+2) including the ghost frame, x fastest."""
    with open(path, "rb") as f:
        buf = f.read()
    tag = buf[:8].rstrip(b"\0").decode()
    (nvec,) = struct.unpack_from("<i", buf, 8)
    dt, time = struct.unpack_from("<dd", buf, 12)
    (rec,) = struct.unpack_from("<i", buf, 28)
    pos = 32
    vecs = []
    for _ in range(nvec):
        nx, ny, nz, ix, iy, iz = struct.unpack_from("<6i", buf, pos)
        pos += 24
        cnt = nx * ny * nz
        a = np.frombuffer(buf, dtype="<f8", count=cnt, offset=pos).reshape(nz, ny, nx).copy()
        pos += 8 * cnt
        vecs.append(((ix, iy, iz), a))
    return {"tag": tag, "dt": dt, "time": time, "recompute": rec, "vectors": vecs}


def list_dumps(directory: str, kind: str):
    return sorted(glob.glob(os.path.join(directory, f"{kind}_*.bin")))
