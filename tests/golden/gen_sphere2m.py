"""Generate tests/golden/sphere2m_lists.json: the trees, effective directions
and interaction lists of the 2,000,000-point sphere workload (unit sphere,
normalised Gaussian samples, seed 0; k = 2 pi 64, order 5, leaf size 64),
computed by the oracle restatement (oracle/defmm_oracle.cpp, itself pinned
bit-exact to the reference on the cases of tests/golden/cases.py) in its
lists-only mode.  The reference itself cannot run here: its precomputation
of this workload needs several hundred GB of host memory.

Pins written:
* SHA-256 digests of both trees (cell records, centres, effective
  directions, particle permutation), as tests/golden/gen_golden.py does;
* order-independent digests (count and two 64-bit sums of per-record
  hashes, oracle.records_digest) of the near list and of the far lists,
  whose records carry the cone of every far pair.

Usage (takes a few minutes and ~20 GB of host memory):
    python tests/golden/gen_sphere2m.py
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from defmm_b200 import workloads as W  # noqa: E402
from tests.golden.gen_golden import digest  # noqa: E402


def main():
    from oracle import oracle as O
    w = W.sphere_surface(2_000_000, seed=0)
    t0 = time.time()
    o = O.OracleFMM(w.points, w.points, w.order, w.ncrit, w.kappa, -1, lists_only=True)
    if o.status:
        raise SystemExit(f"oracle status {o.status}")
    t1 = time.time()
    inf = o.info()
    meta = {"case": "sphere2m", "n": w.n, "order": w.order, "ncrit": w.ncrit, "kappa": w.kappa,
            "tree_T": digest(*o.tree("T")), "tree_S": digest(*o.tree("S")),
            "lists": o.lists_digest(),
            "counts": {k: inf[k] for k in ("nlvl", "cpt", "max_stage", "n_far_hf", "n_far_lf", "n_near",
                                           "cells_T", "cells_S", "nsrc_exp", "ntrg_exp")},
            "oracle_seconds": round(t1 - t0, 1)}
    with open(os.path.join(HERE, "sphere2m_lists.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print(json.dumps(meta["counts"]), "oracle", meta["oracle_seconds"], "s")


if __name__ == "__main__":
    main()
