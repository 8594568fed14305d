"""PFB files of the device state (pfgpu_write_pfb / pfgpu_read_pfb) against
the host PFB reader/writer (parflow_b200/pfb.py), which reads the
reference's own output files in the golden pipeline.

Written files must read back bitwise; files of several subgrids (as ParFlow
writes them from P x Q x R processes) must scatter to the same field; a field
read from a file must give the solve the same field uploaded directly gives;
malformed files are argument errors.
"""

import struct

import numpy as np
import pytest

from parflow_b200 import configs, pfb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _problem():
    return configs.box(nx=20, ny=14, nz=9, nsteps=2, dt=0.1, seed=5)


def _write_subgrids(path, a, splits, dx=1.0, dy=1.0, dz=0.5):
    """PFB with the grid cut into px x py x pz subgrids (x fastest inside each)."""
    nz, ny, nx = a.shape
    px, py, pz = splits
    cut = lambda n, p: [n * q // p for q in range(p + 1)]
    xs, ys, zs = cut(nx, px), cut(ny, py), cut(nz, pz)
    with open(path, "wb") as f:
        f.write(struct.pack(">ddd", 0.0, 0.0, 0.0))
        f.write(struct.pack(">iii", nx, ny, nz))
        f.write(struct.pack(">ddd", dx, dy, dz))
        f.write(struct.pack(">i", px * py * pz))
        for r in range(pz):
            for q in range(py):
                for p in range(px):
                    x0, x1, y0, y1, z0, z1 = xs[p], xs[p + 1], ys[q], ys[q + 1], zs[r], zs[r + 1]
                    f.write(struct.pack(">iiiiiiiii", x0, y0, z0, x1 - x0, y1 - y0, z1 - z0,
                                        p, q, r))
                    f.write(a[z0:z1, y0:y1, x0:x1].astype(">f8").tobytes(order="C"))


def test_write_pressure_roundtrip(solver, tmp_path):
    prob = _problem()
    s = solver.RichardsGPU(prob)
    rng = np.random.default_rng(1)
    p = prob.initial_pressure() + rng.standard_normal(prob.shape)
    s.set_pressure(p)
    path = str(tmp_path / "press.pfb")
    s.write_pfb(path, "pressure", origin=(1.0, 2.0, 3.0))
    got = pfb.read_pfb(path)
    assert np.array_equal(got, p)
    with open(path, "rb") as f:
        hdr = f.read(64)
    assert struct.unpack(">ddd", hdr[:24]) == (1.0, 2.0, 3.0)
    assert struct.unpack(">iii", hdr[24:36]) == (prob.nx, prob.ny, prob.nz)
    assert struct.unpack(">ddd", hdr[36:60]) == (prob.dx, prob.dy, prob.dz)
    s.close()


def test_write_saturation(solver, tmp_path):
    prob = _problem()
    s = solver.RichardsGPU(prob)
    p = prob.initial_pressure()
    s.set_pressure(p)
    path = str(tmp_path / "satur.pfb")
    s.write_pfb(path, "saturation")
    assert np.array_equal(pfb.read_pfb(path), s.saturation(p))
    s.close()


@pytest.mark.parametrize("splits", [(1, 1, 1), (2, 3, 1), (3, 2, 2)])
def test_read_pressure_subgrids(solver, tmp_path, splits):
    prob = _problem()
    s = solver.RichardsGPU(prob)
    a = np.random.default_rng(2).standard_normal(prob.shape)
    path = str(tmp_path / "in.pfb")
    _write_subgrids(path, a, splits)
    s.read_pfb(path, "pressure")
    assert np.array_equal(s.get_pressure(), a)
    s.close()


def test_read_field_matches_upload(solver, tmp_path):
    prob = _problem()
    path = str(tmp_path / "perm.pfb")
    _write_subgrids(path, prob.field3d(prob.perm), (2, 2, 1))
    ref = solver.RichardsGPU(prob)
    ref.set_pressure(prob.initial_pressure())
    ref.advance(2, prob.dt)
    want = ref.get_pressure()
    ref.close()
    other = _problem()
    other.perm = np.full(other.shape, 0.5)  # replaced by the file's field below
    s = solver.RichardsGPU(other)
    s.read_pfb(path, "perm_x")
    s.set_pressure(prob.initial_pressure())
    s.advance(2, prob.dt)
    assert np.array_equal(s.get_pressure(), want)
    s.close()


def test_read_errors(solver, tmp_path):
    from parflow_b200 import lib as L

    prob = _problem()
    s = solver.RichardsGPU(prob)
    wrong = str(tmp_path / "wrong.pfb")
    pfb.write_pfb(wrong, np.zeros((prob.nz, prob.ny, prob.nx + 1)))
    with pytest.raises(L.PfgpuError):
        s.read_pfb(wrong)
    with pytest.raises(L.PfgpuError):
        s.read_pfb(str(tmp_path / "missing.pfb"))
    short = str(tmp_path / "short.pfb")
    pfb.write_pfb(short, np.zeros(prob.shape))
    with open(short, "r+b") as f:
        f.truncate(200)
    with pytest.raises(L.PfgpuError):
        s.read_pfb(short)
    s.close()
