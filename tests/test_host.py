"""Host-side logic on CPU: file formats, boundary tables, time stepping plan,
layout helpers and the C-ABI surface of libpfgpu.so (no GPU calls)."""

import ctypes
import os
import re

import numpy as np
import pytest

from parflow_b200 import cases, configs
from parflow_b200.pfb import read_pfb, write_pfb
from parflow_b200.pfidb import read_pfidb, write_pfidb
from parflow_b200.problem import BC, BC_DIRICHLET, BC_FLUX, RichardsProblem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pfb_roundtrip(tmp_path):
    a = np.random.default_rng(0).standard_normal((3, 4, 5))
    write_pfb(str(tmp_path / "a.pfb"), a, 1.0, 2.0, 0.5, dist=True)
    assert np.array_equal(read_pfb(str(tmp_path / "a.pfb")), a)
    assert open(str(tmp_path / "a.pfb.dist")).read().strip() == "0"


def test_pfb_reads_reference_layout():
    """Header and big-endian layout of write_parflow_binary.c:74-205."""
    import struct

    g = os.path.join(ROOT, "tests", "golden", "box_small.npz")
    press = np.load(g)["press"][0]
    buf = struct.pack(">ddd", 0, 0, 0) + struct.pack(">iii", 12, 10, 8) + \
        struct.pack(">ddd", 1, 1, 0.5) + struct.pack(">i", 2)
    buf += struct.pack(">9i", 0, 0, 0, 12, 10, 4, 0, 0, 0) + press[:4].astype(">f8").tobytes()
    buf += struct.pack(">9i", 0, 0, 4, 12, 10, 4, 0, 0, 0) + press[4:].astype(">f8").tobytes()
    import tempfile

    with tempfile.NamedTemporaryFile(suffix=".pfb", delete=False) as f:
        f.write(buf)
    assert np.array_equal(read_pfb(f.name), press)
    os.unlink(f.name)


def test_pfidb_roundtrip(tmp_path):
    keys = {"A.B": 1, "C": 0.1, "D.E.F": "x y", "G": True}
    write_pfidb(keys, str(tmp_path / "r.pfidb"))
    back = read_pfidb(str(tmp_path / "r.pfidb"))
    assert back == {"A.B": "1", "C": "0.1", "D.E.F": "x y", "G": "True"}
    lines = open(str(tmp_path / "r.pfidb")).read().split("\n")
    assert lines[0] == "4" and lines[1] == "3" and lines[2] == "A.B"


def test_to_reference_keys(tmp_path):
    p = cases.hetero_small()
    run = p.to_reference(str(tmp_path), "r")
    k = read_pfidb(str(tmp_path / (run + ".pfidb")))
    assert k["Solver.Linear.Preconditioner"] == "MGSemi"
    assert k["Phase.Saturation.VanGenuchten.File"] == "1"
    assert k["Patch.z_lower.BCPressure.Type"] == "DirEquilRefPatch"
    assert k["Patch.z_upper.BCPressure.i0.Value"] == "-0.05"
    for f in ("perm.pfb", "vg_alpha.pfb", "ic_press.pfb"):
        assert os.path.exists(str(tmp_path / f)) and os.path.exists(str(tmp_path / (f + ".dist")))
    assert np.array_equal(read_pfb(str(tmp_path / "perm.pfb")), p.perm)


def test_hydrostatic_ic_and_dirichlet_values():
    p = configs.box(nx=4, ny=3, nz=6)
    rsz = p.rsz()
    assert np.allclose(rsz, 0.25 + 0.5 * np.arange(6))
    ic = p.hydrostatic_ic(2.0)
    assert np.array_equal(ic[:, 0, 0], 2.0 - (rsz - 0.0))
    bcs = p.bc_values(0.1)
    typ, bottom = bcs[4]
    assert typ == BC_DIRICHLET and np.all(bottom == 2.0)   # z = 0 on the bottom face
    typ, top = bcs[5]
    assert typ == BC_FLUX and np.all(top == -0.05)


def test_time_cycle_intervals():
    """time_cycle_data.c:153-199: discretised time, 1-based interval end."""
    bc = BC(BC_FLUX, (-0.01, 0.0), lengths=(8, 8), repeat=-1)
    vals = [bc.value_at(0.25 * (s + 1), 0.25, 0.0) for s in range(20)]
    assert vals[:8] == [-0.01] * 8 and vals[8:16] == [0.0] * 8 and vals[16:] == [-0.01] * 4


def test_time_plan_last_step_snaps_to_stop():
    p = cases.box_odd()
    plan = p.time_plan()
    assert len(plan) == 3
    assert plan[0] == (0.1, 0.1) and plan[1] == (0.2, 0.1)
    t3, dt3 = plan[2]
    assert t3 == p.stop_time() and dt3 == p.stop_time() - 0.2 and dt3 != 0.1


def test_pad_unpad():
    from parflow_b200.solver import pad, unpad

    a = np.arange(24.0).reshape(2, 3, 4)
    b = pad(a)
    assert b.shape == (4, 5, 6) and b[0].sum() == 0 and np.array_equal(unpad(b), a)
    # ParFlow SubvectorEltIndex with ix=iy=iz=-1
    flat = b.ravel()
    for (k, j, i) in [(0, 0, 0), (1, 2, 3)]:
        assert flat[(i + 1) + ((j + 1) + (k + 1) * 5) * 6] == a[k, j, i]


def _header_symbols():
    src = open(os.path.join(ROOT, "include", "pfgpu.h")).read()
    return sorted(set(re.findall(r"\b(pfgpu_[a-z_]+)\s*\(", src)))


def test_lib_exports_every_header_symbol():
    """libpfgpu.so loads (no GPU call) and exports each declared entry point."""
    from parflow_b200 import lib

    path = lib.LIB_PATH
    if not os.path.exists(path):
        pytest.fail("libpfgpu.so missing: run __graft_entry__.build()")
    L = ctypes.CDLL(path)
    syms = _header_symbols()
    assert len(syms) >= 17
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) <= set(lib.EXPORTS)


def test_create_rejects_bad_descriptor():
    """Argument checks run before any CUDA call."""
    from parflow_b200 import lib

    L = lib.load()
    d = lib.Desc()
    d.abi_version = 999
    assert not L.pfgpu_create(ctypes.byref(d), 0)
    assert "ABI" in lib.last_error()
    d.abi_version = lib.ABI_VERSION
    d.nx = d.ny = d.nz = 1
    assert not L.pfgpu_create(ctypes.byref(d), 0)
    assert "two cells" in lib.last_error()


def test_ensemble_members_seeded_and_in_range():
    """Config-3 members: sizes from the stated sets, parameters in their
    ranges, the same member twice is the same problem."""
    from parflow_b200 import configs

    ms = configs.ensemble(48)
    assert len(ms) == 48
    for m in ms:
        assert m.nx == m.ny and m.nx in configs.ENSEMBLE_NXY and m.nz in configs.ENSEMBLE_NZ
        assert 0.5 <= m.vg_alpha <= 4.0 and 1.4 <= m.vg_n <= 3.0
        assert -0.1 <= m.bc["z_upper"].values[0] <= -0.02
    a, b = configs.ensemble_member(7), configs.ensemble_member(7)
    assert np.array_equal(a.perm, b.perm) and a.vg_alpha == b.vg_alpha
    assert len({(m.nx, m.nz) for m in ms}) > 4  # uneven sizes
