"""Generates the golden fixtures in tests/golden/ by running the reference
ParFlow build (oracle/_ref/bin/parflow_hook, built by oracle/ref.mk from the
unmodified reference sources) on small seeded Richards problems.

Each fixture ``<case>.npz`` holds the problem's input fields, the pressure
after every timestep as written by the reference (PFB output), the per-step
KINSOL counters from ``<run>.out.kinsol.log``, and a few operand dumps of the
reference's own KINSolFunctionEval / KINSolMatVec / KinsolPC calls
(interior cells).  Run from the repository root:

    make -f oracle/ref.mk -j8 seq REF=<parflow source tree>
    python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.refdump import list_dumps, read_dump  # noqa: E402
from parflow_b200 import cases  # noqa: E402
from parflow_b200.pfb import read_pfb  # noqa: E402

HOOK = os.path.join(ROOT, "oracle", "_ref", "bin", "parflow_hook")
OUT = os.path.dirname(os.path.abspath(__file__))


def kinsol_counts(log: str):
    keys = ["Nonlin. Its.", "Lin. Its.", "Func. Evals.", "PC Evals.", "PC Solves",
            "Lin. Conv. Fails", "Beta Cond. Fails", "Backtracks"]
    rows = []
    for block in log.split("KINSOL starting step")[1:]:
        vals = []
        for k in keys:
            m = re.search(re.escape(k) + r":?\s+(\d+)", block)
            vals.append(int(m.group(1)) if m else -1)
        rows.append(vals)
    return np.array(rows, dtype=np.int64)


def attempt_times(log: str):
    """Target time of every nonlinear solve in a kinsol.log, in order (a
    solve that failed is followed by a retry at an earlier time)."""
    return np.array([float(x) for x in re.findall(r"KINSOL starting step for time ([-+0-9.eE]+)",
                                                  log)])


def make(case_name: str, max_dumps: int = 6):
    prob = cases.get(case_name)
    with tempfile.TemporaryDirectory() as wd:
        run = prob.to_reference(wd, "golden", dump_interval=cases.DUMP.get(case_name, 1))
        dump = os.path.join(wd, "dump")
        os.makedirs(dump)
        env = dict(os.environ, PFREF_DUMP_DIR=dump, PFREF_DUMP_MAX=str(max_dumps))
        subprocess.run([HOOK, run], cwd=wd, env=env, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        nfiles = 0
        while os.path.exists(os.path.join(wd, f"{run}.out.press.{nfiles:05d}.pfb")):
            nfiles += 1
        press = np.stack([read_pfb(os.path.join(wd, f"{run}.out.press.{t:05d}.pfb"))
                          for t in range(nfiles)])
        log = open(os.path.join(wd, f"{run}.out.kinsol.log")).read()
        counts = kinsol_counts(log)
        inner = lambda a: np.ascontiguousarray(a[1:-1, 1:-1, 1:-1])

        def stack(arrs):
            return np.stack(arrs) if arrs else np.zeros((0,) + prob.shape)
        # face velocities (and overland fluxes) after every step, where the
        # case prints them (Solver.PrintVelocities / PrintQ{x,y}Overland)
        extra = {}
        for key, tag in (("velx", "velx"), ("vely", "vely"), ("velz", "velz"),
                         ("qx_overland", "qx_overland"), ("qy_overland", "qy_overland")):
            files = [os.path.join(wd, f"{run}.out.{tag}.{t:05d}.pfb")
                     for t in range(1, nfiles)]
            if all(os.path.exists(f) for f in files):
                extra[key] = np.stack([read_pfb(f) for f in files])
        if prob.evap_trans is not None:
            extra["evap_trans"] = prob.field3d(prob.evap_trans)
        out = {"press": press, "counts": counts, "attempt_times": attempt_times(log), **extra,
               "perm": prob.field3d(prob.perm), "alpha": prob.field3d(prob.vg_alpha),
               "n": prob.field3d(prob.vg_n)}
        fe = [read_dump(f) for f in list_dumps(dump, "fe")]
        out["fe_p"] = stack([inner(d["vectors"][0][1]) for d in fe])
        out["fe_f"] = stack([inner(d["vectors"][1][1]) for d in fe])
        out["fe_pold"] = stack([inner(d["vectors"][4][1]) for d in fe])
        out["fe_sold"] = stack([inner(d["vectors"][5][1]) for d in fe])
        out["fe_dt"] = np.array([d["dt"] for d in fe])
        out["fe_time"] = np.array([d["time"] for d in fe])
        mv = [read_dump(f) for f in list_dumps(dump, "mv")]
        pc = [read_dump(f) for f in list_dumps(dump, "pc")]
        out["mv_x"] = stack([inner(d["vectors"][0][1]) for d in mv])
        out["mv_y"] = stack([inner(d["vectors"][1][1]) for d in mv])
        out["mv_p"] = stack([inner(d["vectors"][2][1]) for d in mv])
        out["mv_pold"] = stack([inner(d["vectors"][3][1]) for d in mv])
        out["mv_dt"] = np.array([d["dt"] for d in mv])
        out["mv_time"] = np.array([d["time"] for d in mv])
        out["pc_in"] = stack([inner(d["vectors"][0][1]) for d in pc])
        out["pc_out"] = stack([inner(d["vectors"][1][1]) for d in pc])
        np.savez_compressed(os.path.join(OUT, f"{case_name}.npz"), **out)
        print(case_name, "steps", prob.nsteps, "counts", counts[:, :2].tolist())


if __name__ == "__main__":
    if not os.path.exists(HOOK):
        sys.exit(f"{HOOK} missing: build it with make -f oracle/ref.mk seq")
    names = sys.argv[1:] or cases.GOLDEN
    for name in names:
        make(name)
