"""ParFlow binary (PFB) field files.

Layout as written by ``WritePFBinary`` (pfsimulator/parflow_lib/write_parflow_binary.c:74-205)
and read by ``ReadPFBinary`` (pfsimulator/parflow_lib/read_parflow_binary.c:38-120), all
big-endian: origin x, y, z (f64); nx, ny, nz (i32); dx, dy, dz (f64); number of
subgrids (i32); then per subgrid ix, iy, iz, nx, ny, nz, rx, ry, rz (i32) followed by
the subgrid's values, x fastest (f64).
"""

from __future__ import annotations

import struct

import numpy as np


def write_pfb(path: str, data: np.ndarray, dx: float = 1.0, dy: float = 1.0,
              dz: float = 1.0, origin=(0.0, 0.0, 0.0), dist: bool = False) -> None:
    """Write a (nz, ny, nx) array as a single-subgrid PFB file.

    ``dist`` also writes the ``<path>.dist`` offset file that ParFlow's
    ``amps_FFopen`` (pfsimulator/amps/common/amps_ffopen.c:243-281) requires
    for input files; with one process it holds the single offset 0."""
    a = np.asarray(data, dtype=np.float64)
    if a.ndim == 2:
        a = a[None, :, :]
    nz, ny, nx = a.shape
    with open(path, "wb") as f:
        f.write(struct.pack(">ddd", *origin))
        f.write(struct.pack(">iii", nx, ny, nz))
        f.write(struct.pack(">ddd", dx, dy, dz))
        f.write(struct.pack(">i", 1))
        f.write(struct.pack(">iiiiiiiii", 0, 0, 0, nx, ny, nz, 0, 0, 0))
        f.write(a.astype(">f8").tobytes(order="C"))
    if dist:
        with open(path + ".dist", "w") as f:
            f.write("0\n")


def read_pfb(path: str) -> np.ndarray:
    """Read a PFB file (any subgrid layout) into a (nz, ny, nx) float64 array."""
    with open(path, "rb") as f:
        buf = f.read()
    pos = 0

    def take(fmt):
        nonlocal pos
        size = struct.calcsize(fmt)
        vals = struct.unpack(fmt, buf[pos:pos + size])
        pos += size
        return vals

    take(">ddd")
    nx, ny, nz = take(">iii")
    take(">ddd")
    (nsg,) = take(">i")
    out = np.zeros((nz, ny, nx), dtype=np.float64)
    for _ in range(nsg):
        ix, iy, iz, snx, sny, snz, _rx, _ry, _rz = take(">iiiiiiiii")
        cnt = snx * sny * snz
        vals = np.frombuffer(buf, dtype=">f8", count=cnt, offset=pos).astype(np.float64)
        pos += 8 * cnt
        out[iz:iz + snz, iy:iy + sny, ix:ix + snx] = vals.reshape(snz, sny, snx)
    return out


__all__ = ["write_pfb", "read_pfb"]
