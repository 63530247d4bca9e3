"""Generates the golden fixtures of tests/golden/*.npz with the CPU oracle.

The reference (Fortran) cannot be built here and ships no vectors for this
path, so these fixtures pin the oracle's own outputs on seeded synthetic
columns; tests/test_oracle_golden.py checks the oracle still reproduces them
and the GPU tests compare the CUDA path against them.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gitm_b200 import abi, synthetic  # noqa: E402
from oracle import oracle  # noqa: E402

CASES = {
    # name: (n_cols, n_alts, seed, n_steps, dt, param overrides, member kwargs)
    "rusanov_default": (8, 50, 11, 1, 2.0, {}, {}),
    "rusanov_3steps_n20": (6, 20, 12, 3, 2.0, {}, {}),
    "rusanov_msis_damping": (6, 30, 13, 2, 2.0, dict(use_msis_bcs=1, use_damping=1, use_coriolis=0),
                             dict(with_lbc=True)),
    "rusanov_log_ions_nofriction": (6, 24, 14, 2, 2.0,
                                    dict(use_improved_ion_advection=0, use_neutral_friction=0,
                                         use_nighttime_ion_bcs=0), {}),
    "rusanov_given_coefficients": (6, 50, 15, 1, 2.0, dict(compute_coefficients=0), {}),
    "ausm_default": (8, 50, 16, 1, 2.0, dict(solver=abi.SOLVER_AUSM), {}),
    "ausm_2steps_log_ions_nofriction": (6, 30, 17, 2, 2.0,
                                        dict(solver=abi.SOLVER_AUSM, use_neutral_friction=0,
                                             use_improved_ion_advection=0), {}),
    "ausm_msis_nocoriolis": (6, 40, 18, 1, 2.0, dict(solver=abi.SOLVER_AUSM, use_msis_bcs=1, use_coriolis=0),
                             dict(with_lbc=True)),
}


def make_case(name):
    n_cols, n_alts, seed, n_steps, dt, over, mkw = CASES[name]
    p = abi.default_params(**over)
    m = synthetic.make_member(n_cols, n_alts, seed=seed, **mkw)
    inp = m.copy()
    st = oracle.advance(m, p, dt, n_steps, nthreads=1)
    return p, inp, m, st, n_steps, dt


def save(name):
    p, inp, out, st, n_steps, dt = make_case(name)
    d = {"n_steps": n_steps, "dt": dt, "status": st}
    for k, v in inp.arrays():
        d["in_" + k] = v
    for k, v in out.arrays():
        d["out_" + k] = v
    d["n_alts"] = inp.n_alts
    d["n_cols"] = inp.n_cols
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)


if __name__ == "__main__":
    oracle.build()
    names = sys.argv[1:] or list(CASES)
    for name in names:
        save(name)
        print("wrote", name)
