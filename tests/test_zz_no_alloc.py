"""pfgpu_residual_noalloc: the allocation-free residual, called through the C
ABI with device buffers, must match pfgpu_nl_function_eval (the handle-based
residual, itself checked against the oracle) on the same inputs, on two calls
in a row and after a call on another grid has reused the static scratch.

Named so that it is collected last: it must also pass after every other GPU
test has run in the same process.
"""

import ctypes as C

import numpy as np
import pytest

from parflow_b200 import cases
from parflow_b200 import lib as L

pytestmark = pytest.mark.gpu

# same kernels on the same inputs: equal up to rounding of reassociated
# constants, far below the residual's own scale
RTOL = 1e-12


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _inputs(name):
    from parflow_b200.solver import RichardsGPU

    prob = cases.get(name)
    gpu = RichardsGPU(prob)
    t, dt = prob.time_plan()[0]
    p_old = prob.initial_pressure()
    rng = np.random.default_rng(5)
    p = p_old + 0.05 * rng.standard_normal(p_old.shape)
    s_old = gpu.saturation(p_old)
    f_ref = gpu.nl_function_eval(p, p_old, s_old, dt)
    return prob, gpu, t, dt, p, p_old, s_old, f_ref


def _noalloc(torch, prob, gpu, t, dt, p, p_old, s_old):
    dev = torch.device("cuda:0")
    as_dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    keep = []
    perm = as_dev(prob.field3d(prob.perm))
    vg = []
    for v in (prob.vg_alpha, prob.vg_n, prob.s_res, prob.s_sat):
        a = prob.field3d(v)
        if prob.vg_from_file() and not np.all(a == a.flat[0]):
            keep.append(as_dev(a))
            vg.append(C.c_void_p(keep[-1].data_ptr()))
        else:
            vg.append(None)
    types = (C.c_int * 6)()
    tables = (C.c_void_p * 6)()
    for face, (typ, vals) in enumerate(prob.bc_values(t)):
        types[face] = typ
        keep.append(as_dev(vals))
        tables[face] = keep[-1].data_ptr()
    dp, dpo, dso = as_dev(p), as_dev(p_old), as_dev(s_old)
    f = torch.full(prob.shape, np.nan, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = L.load().pfgpu_residual_noalloc(
        C.byref(gpu.desc), C.c_void_p(perm.data_ptr()), *vg, types, tables,
        C.c_void_p(dp.data_ptr()), C.c_void_p(dpo.data_ptr()), C.c_void_p(dso.data_ptr()),
        dt, C.c_void_p(f.data_ptr()), C.c_void_p(stream.cuda_stream))
    L.check(rc, "pfgpu_residual_noalloc")
    stream.synchronize()
    return f.cpu().numpy()


def _close(a, b):
    scale = np.max(np.abs(b))
    assert np.all(np.isfinite(a))
    np.testing.assert_allclose(a, b, rtol=RTOL, atol=RTOL * scale)


@pytest.mark.parametrize("name", ["box_odd", "hetero_small", "walker2_small"])
def test_noalloc_residual_matches_handle_twice(name):
    torch = _torch()
    prob, gpu, t, dt, p, p_old, s_old, f_ref = _inputs(name)
    first = _noalloc(torch, prob, gpu, t, dt, p, p_old, s_old)
    second = _noalloc(torch, prob, gpu, t, dt, p, p_old, s_old)
    _close(first, f_ref)
    _close(second, f_ref)
    gpu.close()


def test_noalloc_scratch_reused_across_grids():
    """A call on another grid in between leaves no trace in the next result."""
    torch = _torch()
    a = _inputs("hetero_small")
    b = _inputs("box_odd")
    _close(_noalloc(torch, *a[:7]), a[7])
    _close(_noalloc(torch, *b[:7]), b[7])
    _close(_noalloc(torch, *a[:7]), a[7])
    a[1].close()
    b[1].close()


def test_noalloc_rejects_grid_beyond_scratch():
    """The size check runs on the host before any pointer is touched."""
    _torch()
    prob = cases.get("box_small")
    from parflow_b200.solver import RichardsGPU

    gpu = RichardsGPU(prob)
    d = L.Desc.from_buffer_copy(gpu.desc)
    d.nx, d.ny, d.nz = 128, 128, 32  # 2^19 cells > 2^18
    types = (C.c_int * 6)()
    tables = (C.c_void_p * 6)()
    rc = L.load().pfgpu_residual_noalloc(C.byref(d), None, None, None, None, None, types,
                                         tables, None, None, None, 1.0, None, None)
    assert rc == -1
    assert "exceed" in L.last_error()
    gpu.close()


def test_noalloc_allocates_no_device_memory():
    """Warmed-up calls leave the device's free memory unchanged: the scratch
    is the library's static array, not an allocation made by the call."""
    torch = _torch()
    inp = _inputs("hetero_small")
    _noalloc(torch, *inp[:7])  # warm: the first call resolves the scratch address
    torch.cuda.synchronize()
    # every buffer the calls below use is allocated first; the free-memory
    # bracket holds only the library calls themselves
    prob, gpu, t, dt, p, p_old, s_old, f_ref = inp
    dev = torch.device("cuda:0")
    as_dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    perm = as_dev(prob.field3d(prob.perm))
    keep, vg = [], []
    for v in (prob.vg_alpha, prob.vg_n, prob.s_res, prob.s_sat):
        a = prob.field3d(v)
        if prob.vg_from_file() and not np.all(a == a.flat[0]):
            keep.append(as_dev(a))
            vg.append(C.c_void_p(keep[-1].data_ptr()))
        else:
            vg.append(None)
    types = (C.c_int * 6)()
    tables = (C.c_void_p * 6)()
    for face, (typ, vals) in enumerate(prob.bc_values(t)):
        types[face] = typ
        keep.append(as_dev(vals))
        tables[face] = keep[-1].data_ptr()
    dp, dpo, dso = as_dev(p), as_dev(p_old), as_dev(s_old)
    f = torch.empty(prob.shape, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    for _ in range(3):
        rc = L.load().pfgpu_residual_noalloc(
            C.byref(gpu.desc), C.c_void_p(perm.data_ptr()), *vg, types, tables,
            C.c_void_p(dp.data_ptr()), C.c_void_p(dpo.data_ptr()), C.c_void_p(dso.data_ptr()),
            dt, C.c_void_p(f.data_ptr()), C.c_void_p(stream.cuda_stream))
        L.check(rc, "pfgpu_residual_noalloc")
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(dev)[0]
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    _close(f.cpu().numpy(), f_ref)
    gpu.close()


def test_noalloc_rejects_host_buffers():
    """A host buffer where device memory is required is refused on the host,
    before any kernel is launched."""
    _torch()
    prob = cases.get("box_small")
    from parflow_b200.solver import RichardsGPU

    gpu = RichardsGPU(prob)
    host = np.zeros(prob.ncells)
    hp = C.c_void_p(host.ctypes.data)
    types = (C.c_int * 6)()
    tables = (C.c_void_p * 6)()
    rc = L.load().pfgpu_residual_noalloc(C.byref(gpu.desc), hp, None, None, None, None, types,
                                         tables, hp, hp, hp, 1.0, hp, None)
    assert rc == -1
    assert "current device" in L.last_error()
    gpu.close()
