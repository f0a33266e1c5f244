"""Test infrastructure: runs one FESolver::computePhi of the reference
(oracle/_ref) in a process of its own.

The reference's NonLinear method ends the process with exit(-1) when Newton
fails (src/FESolver.cpp:359-362), so the tests call it here, in a child
process that has touched no GPU, and read its outcome back:

    python -m oracle.ref_isolated <deck_dir> <in.npz> <out.npz>

in.npz holds method, spwt, d, F1, den and optionally fixed_nodes /
fixed_value / fixed_file (an extra Dirichlet surface such as the sphere).
out.npz receives d and uh; the reference's own messages go to stdout/stderr.
"""
from __future__ import annotations

import os
import sys

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref  # noqa: E402


def main(deck_dir: str, inp: str, out: str) -> None:
    a = dict(np.load(inp))
    extra = {}
    if "fixed_file" in a:
        extra = {str(a["fixed_file"]): (a["fixed_nodes"], float(a["fixed_value"]))}
    s = ref.RefSim(deck_dir, spwt=float(a["spwt"]), extra_fixed=extra)
    s.set("d", a["d"])
    s.set("F1", a["F1"])
    s.set("den", a["den"])
    sys.stdout.flush()
    s.compute_phi(int(a["method"]))  # may exit(-1), as the reference does
    np.savez(out, d=s.get("d"), uh=s.get("uh"), F1=s.get("F1"))
    s.close()


if __name__ == "__main__":
    main(*sys.argv[1:4])
