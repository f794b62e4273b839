"""The oracle (C++ restatement of the reference, oracle/defmm_oracle.cpp)
against the reference's own outputs: the golden fixtures made from the
reference by tests/golden/gen_golden.py, and, where the reference build is
present, the reference run directly."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import refrun
from tests.golden.cases import CASES, case_inputs
from tests.golden.gen_golden import digest, pins, sample_index, sort_rows

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FAST = ["cube_lf", "fixed_depth", "blobs_sphere"]


def load(name):
    with open(os.path.join(GOLD, f"{name}.json")) as f:
        meta = json.load(f)
    return meta, np.load(os.path.join(GOLD, f"{name}_pot_sample.npy"))


@pytest.mark.parametrize("name", CASES)
def test_oracle_tree_and_lists_match_reference_digests(name):
    meta, _ = load(name)
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    o = O.OracleFMM(src, trg, L, ncrit, kappa, lvmax)
    assert o.status == 0
    for tag in "TS":
        ci, cd, dirs, perm = o.tree(tag)
        assert digest(ci, cd, dirs, perm) == meta[f"tree_{tag}"], tag
    near, fh, fl = o.lists()
    assert digest(sort_rows(near)) == meta["near"]
    assert digest(sort_rows(fh)) == meta["far_hf"]
    assert digest(sort_rows(fl)) == meta["far_lf"]


@pytest.mark.parametrize("name", FAST + ["cube20k"])
def test_oracle_potentials_match_reference(name):
    meta, sample = load(name)
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    o = O.OracleFMM(src, trg, L, ncrit, kappa, lvmax)
    p = o.gemv(q)
    idx = sample_index(trg.shape[0])
    assert np.linalg.norm(p[idx] - sample) <= 1e-13 * np.linalg.norm(sample)
    got = pins(p)
    ref = meta["pins"]
    scale = np.sqrt(ref["sumsq"])
    assert abs(complex(*got["sum"]) - complex(*ref["sum"])) <= 1e-12 * scale * np.sqrt(len(p))
    assert abs(got["sumsq"] - ref["sumsq"]) <= 1e-12 * ref["sumsq"]
    assert abs(complex(*got["proj"]) - complex(*ref["proj"])) <= 1e-12 * scale * np.sqrt(len(p))


@pytest.mark.skipif(not refrun.available(), reason="reference build (oracle/_ref) absent")
def test_oracle_matches_reference_run_directly():
    from defmm_b200 import workloads as W
    pts = W.sphere_surface(6000, seed=21, wavelengths=12).points
    q = W.charges(6000, 2)
    r = refrun.run(pts, pts, q, 4, 48, 2 * np.pi * 6)
    o = O.OracleFMM(pts, pts, 4, 48, 2 * np.pi * 6)
    assert np.array_equal(o.tree("T")[0], r.T.cells_int)
    assert np.linalg.norm(o.gemv(q) - r.pot) <= 1e-13 * np.linalg.norm(r.pot)


def test_direct_sum_matches_numpy():
    rng = np.random.default_rng(3)
    src = rng.uniform(-1, 1, (300, 3))
    trg = np.concatenate([src[:20], rng.uniform(-1, 1, (30, 3))])
    q = rng.standard_normal(300) + 1j * rng.standard_normal(300)
    k = 7.5
    d = np.linalg.norm(trg[:, None] - src[None], axis=-1)
    with np.errstate(divide="ignore", invalid="ignore"):
        K = np.where(d * d < 1e-16, 0, np.exp(1j * k * d) / (4 * np.pi * d))
    assert np.allclose(O.direct(src, q, trg, k), K @ q, rtol=1e-13, atol=0)


def test_oracle_planted_mistake_is_detected():
    # a mistake planted in the checker's input (one charge changed) must move
    # the potentials well beyond the parity tolerance
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_lf")
    o = O.OracleFMM(src, trg, L, ncrit, kappa, lvmax)
    p = o.gemv(q)
    q2 = q.copy()
    q2[123] += 1e-6
    p2 = o.gemv(q2)
    assert np.linalg.norm(p2 - p) > 1e-10 * np.linalg.norm(p)
