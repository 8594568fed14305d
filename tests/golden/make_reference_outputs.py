"""Copies a few of the reference's own regression outputs into a fixture:
test/correct_output/default_richards.out.{press,satur}.NNNNN.pfb of the
ParFlow source tree (made by test/python/default_richards.py with the PFMG
preconditioner) at steps 1, 10, 25 and 50, as tests/golden/default_richards_ref.npz.

    python tests/golden/make_reference_outputs.py <parflow source tree>
"""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from parflow_b200.pfb import read_pfb  # noqa: E402

STEPS = [1, 10, 25, 50]


def main(src: str):
    d = os.path.join(src, "test", "correct_output")
    out = {"steps": np.array(STEPS)}
    for what in ("press", "satur"):
        out[what] = np.stack([read_pfb(os.path.join(d, f"default_richards.out.{what}.{s:05d}.pfb"))
                              for s in STEPS])
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                     "default_richards_ref.npz"), **out)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PARFLOW_REF_SRC")
    if not src:
        sys.exit("usage: make_reference_outputs.py <parflow source tree> "
                 "(or set PARFLOW_REF_SRC)")
    main(src)
