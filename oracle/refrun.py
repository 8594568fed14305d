"""Test and benchmark infrastructure: runs the unmodified reference CPU build
(oracle/_ref/bin/parflow or parflow_omp, made by oracle/ref.mk from the
ParFlow sources) on a RichardsProblem and times every timestep.

Per-step times come from the reference's own KINSOL log: KinsolNonlinSolver
prints its per-step counters at the end of every nonlinear solve and flushes
the file (pfsimulator/parflow_lib/kinsol_nonlin_solver.c:240-262), so a
thread that polls the log sees step s end within the polling interval.  The
binary is run as built; nothing is linked into it for timing.

Used only by tests/ and bench.py's CPU legs (the reference arm and the CPU
baseline), never by the library.
"""

from __future__ import annotations

import os
import re
import shutil
import subprocess
import tempfile
import threading
import time
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "bin")
_KEYS = ["Nonlin. Its.", "Lin. Its.", "Func. Evals.", "PC Evals.", "PC Solves",
         "Lin. Conv. Fails", "Beta Cond. Fails", "Backtracks"]
_END = "Backtracks:"  # last line of a step's counter block


def binary(name: str = "parflow_omp") -> Optional[str]:
    p = os.path.join(BIN, name)
    return p if os.path.exists(p) else None


def kinsol_counts(log: str) -> np.ndarray:
    """Per-step KINSOL counters (rows: steps; columns: _KEYS) of a kinsol.log."""
    rows = []
    for block in log.split("KINSOL starting step")[1:]:
        vals = []
        for k in _KEYS:
            m = re.search(re.escape(k) + r":?\s+(\d+)", block)
            vals.append(int(m.group(1)) if m else -1)
        rows.append(vals)
    return np.array(rows, dtype=np.int64).reshape(-1, len(_KEYS))


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class _LogWatch(threading.Thread):
    """Records the wall time at which each step's counter block appears."""

    def __init__(self, path: str, t0: float, poll: float):
        super().__init__(daemon=True)
        self.path, self.t0, self.poll = path, t0, poll
        self.ends: list = []
        self.stop = threading.Event()

    def scan(self):
        try:
            with open(self.path, "r", errors="replace") as f:
                n = f.read().count(_END)
        except OSError:
            return
        now = time.perf_counter() - self.t0
        while len(self.ends) < n:
            self.ends.append(now)

    def run(self):
        while not self.stop.is_set():
            self.scan()
            self.stop.wait(self.poll)
        self.scan()


def run(prob, nsteps: int, exe: str = "parflow_omp", threads: Optional[int] = None,
        dump: bool = False, workdir: Optional[str] = None, poll: float = 0.02,
        keep: bool = False) -> dict:
    """Run the reference on ``prob`` for ``nsteps`` timesteps of prob.dt.

    Returns a dict with the total wall time (``wall``, from process start to
    exit), the wall time at the end of every step (``step_end``, from process
    start; the first entry includes input reading and set-up), the per-step
    KINSOL counters (``counts``), the module times of the reference's timing
    file (``timing``), the pressure after every step when ``dump`` is set
    (``press``, interior cells, shape (nsteps, nz, ny, nx)), and the binary
    and thread count used."""
    from parflow_b200.pfb import read_pfb

    path = binary(exe)
    if path is None:
        raise FileNotFoundError(f"reference build {exe} missing under {BIN}")
    saved = prob.nsteps
    prob.nsteps = nsteps
    wd = workdir or tempfile.mkdtemp(prefix="pfref_")
    try:
        name = prob.to_reference(wd, "ref", dump_interval=1 if dump else 0)
        threads = threads or (os.cpu_count() or 1)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        log = os.path.join(wd, name + ".out.kinsol.log")
        t0 = time.perf_counter()
        watch = _LogWatch(log, t0, poll)
        watch.start()
        proc = subprocess.run([path, name], cwd=wd, env=env, stdout=subprocess.PIPE,
                              stderr=subprocess.STDOUT, text=True)
        wall = time.perf_counter() - t0
        watch.stop.set()
        watch.join()
        if proc.returncode != 0:
            raise RuntimeError(f"reference run failed ({proc.returncode}): {proc.stdout[-2000:]}")
        counts = kinsol_counts(open(log).read())
        timing = {}
        try:
            for line in open(os.path.join(wd, name + ".out.timing.csv")):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 2:
                    try:
                        timing[parts[0]] = float(parts[1])
                    except ValueError:
                        pass
        except OSError:
            pass
        out = {"wall": wall, "step_end": list(watch.ends), "counts": counts, "timing": timing,
               "binary": exe, "threads": threads if exe == "parflow_omp" else 1}
        if dump:
            out["press"] = np.stack([read_pfb(os.path.join(wd, f"{name}.out.press.{t:05d}.pfb"))
                                     for t in range(1, nsteps + 1)])
        return out
    finally:
        prob.nsteps = saved
        if not keep and workdir is None:
            shutil.rmtree(wd, ignore_errors=True)


def steps_per_second(res: dict, first: int, count: int) -> float:
    """Timesteps/s over steps first+1 .. first+count (0-based step ends): the
    time from the end of step `first` (the process start when first == 0)
    to the end of step first+count."""
    ends = res["step_end"]
    if len(ends) < first + count:
        raise RuntimeError(f"only {len(ends)} step ends recorded, need {first + count}")
    t_a = ends[first - 1] if first > 0 else 0.0
    return count / (ends[first + count - 1] - t_a)
