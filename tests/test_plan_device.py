"""The plan's octree build and level walk on the GPU (plan_device.cu: the
particles ordered level by level with octant codes, counts and a stable
radix sort; the dual traversal with the M2M/L2L transfer lists; the
near-field chunks, symmetric blocks and work items; the transfer spectra and
signatures) against the host build and walk (plan.cpp, itself
pinned to the reference's trees, cones and lists by tests/test_plan.py):
same statistics, same effective directions per cell (the cell-array dump,
which carries the slots' directions), fingerprints of every near-field work
list, and a bit-identical FP64 matvec, which
needs identical slots, far entries, transfer lists and tables in identical
order.
"""
import numpy as np
import pytest

from defmm_b200 import IBFMM_Mat, workloads as W
from tests.golden.cases import CASES, case_inputs

pytestmark = pytest.mark.gpu

STATS = ["nlvl", "cpt", "slots_S", "slots_T", "far_hf", "far_lf", "near", "i_near", "tables",
         "permuted_spectra", "m2l_targets", "leaf_slots_S", "m2m_entries", "l2l_entries"]


def build(src, trg, L, ncrit, kappa, lvmax, device):
    A = IBFMM_Mat()
    A.set_plan_device(device)
    A.addSourceParticles(src)
    A.addTargetParticles(trg)
    A.prcmpt(L, ncrit, kappa, lvmax)
    return A


def compare(src, trg, q, L, ncrit, kappa, lvmax):
    H = build(src, trg, L, ncrit, kappa, lvmax, False)
    D = build(src, trg, L, ncrit, kappa, lvmax, True)
    assert H.info("plan_walk_device") == 0 and D.info("plan_walk_device") == 1
    assert H.info("tree_device") == 0 and D.info("tree_device") == 1
    for k in STATS:
        assert H.info(k) == D.info(k), k
    # near-field lists built on the device, element for element the host's
    assert np.array_equal(H.near_digest(), D.near_digest())
    for which in ("T", "S"):
        for a, b in zip(H.tree(which), D.tree(which)):
            assert np.array_equal(a, b)
    assert np.array_equal(H.matvec(q), D.matvec(q))


@pytest.mark.parametrize("name", CASES)
def test_device_walk_equals_host_walk(name, gpu):
    compare(*case_inputs(name))


def test_device_walk_equals_host_walk_high_frequency_sphere(gpu):
    # deeper HF hierarchy (more direction stages, propagation of effective
    # directions over several levels)
    w = W.sphere_surface(120_000, seed=11, wavelengths=32)
    compare(w.points, w.points, W.charges(w.n, 2), 5, 64, w.kappa, -1)
