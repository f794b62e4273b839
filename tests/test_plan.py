"""The product's host plan (trees, cones, effective directions, lists) is
bit-exact with the reference: against the oracle and the golden digests.
prcmpt runs on the host, so these tests need no GPU."""
import json
import os

import numpy as np
import pytest

from defmm_b200 import IBFMM_Mat, DefmmError, workloads as W
from oracle import oracle as O
from tests.golden.cases import CASES, case_inputs
from tests.golden.gen_golden import digest, sort_rows

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def plan(src, trg, L, ncrit, kappa, lvmax=-1, lists=True):
    A = IBFMM_Mat()
    if lists:
        A.keep_lists()
    A.addSourceParticles(src)
    A.addTargetParticles(trg)
    A.prcmpt(L, ncrit, kappa, lvmax)
    return A


@pytest.mark.parametrize("name", CASES)
def test_plan_matches_reference_digests(name):
    with open(os.path.join(GOLD, f"{name}.json")) as f:
        meta = json.load(f)
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    A = plan(src, trg, L, ncrit, kappa, lvmax)
    for tag in "TS":
        assert digest(*A.tree(tag)) == meta[f"tree_{tag}"], tag
    near, fh, fl = A.lists()
    assert digest(sort_rows(near)) == meta["near"]
    assert digest(sort_rows(fh)) == meta["far_hf"]
    assert digest(sort_rows(fl)) == meta["far_lf"]
    assert A.info("far_hf") == meta["counts"]["far_hf"]


@pytest.mark.parametrize("seed,wl,L,ncrit", [(31, 10, 4, 20), (32, 3, 3, 16), (33, 24, 5, 64)])
def test_plan_matches_oracle_random(seed, wl, L, ncrit):
    pts = W.sphere_surface(12000, seed=seed, wavelengths=wl).points
    pts[::7] *= 0.7  # break the surface symmetry
    kappa = 2 * np.pi * wl / 2
    A = plan(pts, pts, L, ncrit, kappa)
    o = O.OracleFMM(pts, pts, L, ncrit, kappa)
    for tag in "TS":
        for a, b in zip(A.tree(tag), o.tree(tag)):
            assert np.array_equal(a, b)
    for a, b in zip(A.lists(), o.lists()):
        assert np.array_equal(sort_rows(a), sort_rows(b))


@pytest.mark.parametrize("same", [True, False])
def test_near_digest_counts_and_determinism(same):
    # the fingerprints of the near-field work lists (defmm_near_digest, the
    # host build here): its counts are the plan's, and a rebuild repeats
    # every array; distinct targets have no symmetric blocks (empty arrays)
    pts = W.sphere_surface(8000, seed=5, wavelengths=6).points
    trg = pts if same else W.sphere_surface(7000, seed=6, wavelengths=6).points * 0.9
    kappa = 2 * np.pi * 3
    A = plan(pts, trg, 4, 32, kappa, lists=False)
    B = plan(pts, trg, 4, 32, kappa, lists=False)
    da, db = A.near_digest(), B.near_digest()
    assert np.array_equal(da, db)
    assert int(da[25]) == A.info("near") and int(da[24]) == A.info("i_near")
    empty = 1469598103934665603  # FNV-1a of a zero count (8 zero bytes) and no elements
    for _ in range(8):
        empty = (empty * 1099511628211) % (1 << 64)
    for k in range(8, 23):  # own-leaf, symmetric and reduction arrays
        assert (int(da[k]) == empty) == (not same), k


def test_cones_use_first_pair_in_depth_first_order():
    # a lattice: many pairs share a translation; cones must be the ones of
    # the first pair in the reference's traversal (M2L.hpp:189-197)
    g = np.stack(np.meshgrid(*[np.linspace(-0.5, 0.5, 26)] * 3, indexing="ij"), -1).reshape(-1, 3)
    A = plan(g, g, 3, 8, 2 * np.pi * 8)
    o = O.OracleFMM(g, g, 3, 8, 2 * np.pi * 8)
    assert np.array_equal(sort_rows(A.lists()[1]), sort_rows(o.lists()[1]))


def test_empty_input_is_an_error():
    A = IBFMM_Mat()
    with pytest.raises(DefmmError) as e:
        A.prcmpt(4, 32, 1.0)
    assert e.value.code == -1


def test_coincident_points_are_an_error_not_a_hang():
    pts = np.zeros((100, 3))
    pts[50:] = 1.0
    A = IBFMM_Mat()
    A.addSourceParticles(pts)
    A.addTargetParticles(pts)
    with pytest.raises(DefmmError) as e:
        A.prcmpt(4, 32, 5.0)
    assert e.value.code == -2


def test_shallow_tree_is_an_error():
    # fewer points than the leaf size: one level, no M2L level
    # (frequency.hpp:114-120 exits; here a status code)
    pts = W.sphere_surface(20, seed=1).points
    A = IBFMM_Mat()
    A.addSourceParticles(pts)
    A.addTargetParticles(pts)
    with pytest.raises(DefmmError) as e:
        A.prcmpt(4, 64, 50.0)
    assert e.value.code == -3


def test_bad_order_is_an_error():
    pts = W.sphere_surface(2000, seed=1).points
    A = IBFMM_Mat()
    A.addSourceParticles(pts)
    A.addTargetParticles(pts)
    with pytest.raises(DefmmError):
        A.prcmpt(9, 32, 10.0)


def test_inp_loader_reads_xyz_lines(tmp_path):
    pts = W.cube_surface(3000, seed=4).points
    f = tmp_path / "pts.inp"
    np.savetxt(f, pts, fmt="%.17g")
    A = IBFMM_Mat()
    A.addSourceParticlesINP(str(f), len(pts))
    A.addTargetParticlesINP(str(f), len(pts))
    A.prcmpt(4, 32, 2 * np.pi * 6)
    B = plan(pts, pts, 4, 32, 2 * np.pi * 6, lists=False)
    assert np.array_equal(A.tree("S")[1], B.tree("S")[1])
    with pytest.raises(DefmmError) as e:
        IBFMM_Mat().addSourceParticlesINP(str(f), len(pts) + 1)
    assert e.value.code == -6


def test_single_particle_adds_match_bulk():
    pts = W.cube_surface(2000, seed=8).points
    A = IBFMM_Mat()
    for p in pts:
        A.addSourceParticle(p)
        A.addTargetParticle(p)
    A.prcmpt(3, 24, 20.0)
    B = plan(pts, pts, 3, 24, 20.0, lists=False)
    for a, b in zip(A.tree("T"), B.tree("T")):
        assert np.array_equal(a, b)


def test_gemv_without_device_fails_loudly():
    from defmm_b200 import api
    if api.device_count() > 0:
        pytest.skip("a device is present")
    pts = W.cube_surface(2000, seed=8).points
    A = plan(pts, pts, 3, 24, 20.0, lists=False)
    with pytest.raises(DefmmError) as e:
        A.matvec(np.ones(len(pts), complex))
    assert e.value.code == -4
