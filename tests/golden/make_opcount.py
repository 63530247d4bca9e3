"""Counts the FP64 operations of one RK4 column step with the oracle's
instrumented scalar (oracle/flop_counter.hpp) and writes opcount.json.

Convention: + - * / and sqrt count 1 flop each, every exp / log / pow / cos
/ tanh counts 20 flop-equivalents; comparisons, min/max and abs count 0.
Dead code of the reference is not counted (the oracle omits it).  bench.py
reads the file for the roofline's algorithmic flops per column-step.

    python tests/golden/make_opcount.py
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gitm_b200 import abi, synthetic  # noqa: E402
from oracle import oracle  # noqa: E402

TRANS_FLOPS = 20


def count(n_alts=50, seed=1, **over):
    p = abi.default_params(**over)
    m = synthetic.make_member(1, n_alts, seed=seed)
    ops = oracle.count_ops(synthetic.to_modvertical(m, p), p, 2.0)
    flops = ops["add"] + ops["mul"] + ops["div"] + ops["sqrt"] + TRANS_FLOPS * ops["trans"]
    return ops, flops


def main():
    out = {"convention": "add/sub/mul/div/sqrt = 1, transcendental = %d" % TRANS_FLOPS,
           "rusanov": {}, "ausm": {}}
    for name, solver in (("rusanov", abi.SOLVER_RUSANOV), ("ausm", abi.SOLVER_AUSM)):
        for n_alts in (50, 75, 100):
            ops, flops = count(n_alts, solver=solver)
            out[name][str(n_alts)] = {"ops": ops, "flop_eq_per_column_step": flops}
    with open(os.path.join(HERE, "opcount.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
