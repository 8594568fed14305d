"""The two launch forms of the residual kernel give the same F bit for bit:
the gather form (the default: every cell evaluates all six of its faces) and
the face-once form (PFGPU_RESIDUAL_FACE_ONCE=1: each interior face flux
evaluated once, shared through shared memory within a tile and through a
register between planes).  The form is chosen once per process, so each side
runs in a child process.  The Jacobian launches follow the same switch: the
test compares J x and the preconditioner output M^-1 r too."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from parflow_b200 import cases

pytestmark = pytest.mark.gpu

NAMES = ["box_odd", "hetero_small", "walker2_small", "overland_small", "overland_diff_small",
         "overland_flow_small", "tfg_small", "seepage_small", "vel_small"]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from parflow_b200 import cases
from parflow_b200.solver import RichardsGPU
out = {}
for name in json.loads(sys.argv[2]):
    prob = cases.get(name)
    g = RichardsGPU(prob)
    t, dt = prob.time_plan()[0]
    g.set_time(t)
    p_old = prob.initial_pressure()
    p = p_old + 0.03 * np.random.default_rng(3).standard_normal(p_old.shape)
    f = g.nl_function_eval(p, p_old, g.saturation(p_old), dt)
    v = g.face_velocities(dt, p=p, p_old=p_old, s_old=g.saturation(p_old))
    x = np.random.default_rng(4).standard_normal(p.shape)
    y = g.jacobian_matvec(p, dt, x, p_old=p_old)
    g.pc_setup(p, dt, p_old=p_old)
    z = g.pc_apply(x)
    out[name] = [a.tobytes().hex() for a in (f,) + tuple(v) + (y, z)]
    g.close()
json.dump(out, open(sys.argv[3], "w"))
"""


def _run(tmp_path, gather):
    path = str(tmp_path / ("gather.json" if gather else "once.json"))
    env = dict(os.environ)
    if gather:
        env.pop("PFGPU_RESIDUAL_FACE_ONCE", None)
    else:
        env["PFGPU_RESIDUAL_FACE_ONCE"] = "1"
    subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(NAMES), path], env=env,
                   check=True, timeout=600)
    return json.load(open(path))


def test_face_once_equals_gather(tmp_path):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    once = _run(tmp_path, False)
    gather = _run(tmp_path, True)
    for name in NAMES:
        for q, (a, b) in enumerate(zip(once[name], gather[name])):
            if a != b:
                x = np.frombuffer(bytes.fromhex(a))
                y = np.frombuffer(bytes.fromhex(b))
                pytest.fail(f"{name} output {q}: max diff {np.abs(x - y).max()}")
