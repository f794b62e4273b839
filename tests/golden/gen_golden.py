"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the unmodified reference defmm (oracle/_ref/defmm_ref, built by
`make -C oracle ref` from the read-only reference checkout) on seeded
synthetic cases and stores, per case, compact pins of what it produced:

* SHA-256 digests of both trees (cell records, centres, effective
  directions, particle permutation) and of the sorted near / far lists
  (far records carry the cone of each pair);
* the potentials at 500 seeded sample indices, plus three full-vector
  checksums (sum, sum of squared moduli, a seeded random projection).

Usage (in the container that has the reference checkout):
    python tests/golden/gen_golden.py [case ...]   # default: every case
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.cases import CASES, case_inputs  # noqa: E402


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def sort_rows(a):
    return a[np.lexsort(a.T[::-1])] if len(a) else a


def pins(pot):
    rng = np.random.default_rng(12345)
    w = rng.standard_normal(pot.shape[0]) + 1j * rng.standard_normal(pot.shape[0])
    return {"sum": [float(pot.sum().real), float(pot.sum().imag)],
            "sumsq": float(np.sum(np.abs(pot) ** 2)),
            "proj": [float((w * pot).sum().real), float((w * pot).sum().imag)]}


def sample_index(n, m=500):
    return np.sort(np.random.default_rng(777).choice(n, size=min(m, n), replace=False))


def main(names):
    from oracle import refrun
    for name in names:
        src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
        r = refrun.run(src, trg, q, L, ncrit, kappa, lvmax)
        idx = sample_index(trg.shape[0])
        meta = {
            "case": name,
            "tree_T": digest(r.T.cells_int, r.T.cells_dbl, r.T.dirs, r.T.perm),
            "tree_S": digest(r.S.cells_int, r.S.cells_dbl, r.S.dirs, r.S.perm),
            "near": digest(sort_rows(r.near)),
            "far_hf": digest(sort_rows(r.far_hf)),
            "far_lf": digest(sort_rows(r.far_lf)),
            "counts": {"cells_T": int(r.T.cells_int.shape[0]), "cells_S": int(r.S.cells_int.shape[0]),
                       "near": int(r.near.shape[0]), "far_hf": int(r.far_hf.shape[0]),
                       "far_lf": int(r.far_lf.shape[0])},
            "pins": pins(r.pot),
            "reference_gemv_s": r.summary.get("gemv_s"),
        }
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(meta, f, indent=1, sort_keys=True)
        np.save(os.path.join(HERE, f"{name}_pot_sample.npy"), r.pot[idx])
        print(name, meta["counts"], "gemv", meta["reference_gemv_s"])


if __name__ == "__main__":
    main(sys.argv[1:] or CASES)
