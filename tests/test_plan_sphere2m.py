"""Config-2 scale pin: the 2,000,000-point sphere workload (k = 2 pi 64,
order 5, leaf size 64; 9 levels, 368M far pairs).  Its trees, effective
directions and interaction lists (far records with their cones) are
compared with the oracle restatement's, recorded as digests in
tests/golden/sphere2m_lists.json by tests/golden/gen_sphere2m.py: bit-exact
at full size, not only on the small golden cases.

The host-plan test runs without a GPU (about a minute and ~20 GB of host
memory); the GPU test builds the plan with the level walk on the device and
compares it with the same pins and with the host walk's M2L work."""
import json
import os

import numpy as np
import pytest

from defmm_b200 import IBFMM_Mat, workloads as W
from oracle import oracle as O
from tests.golden.gen_golden import digest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def meta():
    with open(os.path.join(GOLD, "sphere2m_lists.json")) as f:
        return json.load(f)


def build(device, lists):
    w = W.sphere_surface(2_000_000, seed=0)
    A = IBFMM_Mat()
    A.set_plan_device(device)
    if lists:
        A.keep_lists()
    A.addSourceParticles(w.points)
    A.addTargetParticles(w.points)
    A.prcmpt(w.order, w.ncrit, w.kappa)
    return A


def check_counts(A, m):
    c = m["counts"]
    assert A.info("nlvl") == c["nlvl"] and A.info("cpt") == c["cpt"] and A.info("max_stage") == c["max_stage"]
    assert A.info("far_hf") == c["n_far_hf"] and A.info("far_lf") == c["n_far_lf"] and A.info("near") == c["n_near"]
    assert A.info("cells_T") == c["cells_T"] and A.info("cells_S") == c["cells_S"]
    assert A.info("slots_S") == c["nsrc_exp"] and A.info("slots_T") == c["ntrg_exp"]


def test_sphere2m_host_plan_is_bit_exact_with_oracle():
    m = meta()
    A = build(False, True)
    check_counts(A, m)
    for tag in "TS":
        assert digest(*A.tree(tag)) == m[f"tree_{tag}"], tag
    near, fh, fl = A.lists()
    assert O.records_digest(near) == m["lists"]["near"]
    del near
    assert O.records_digest(fh) == m["lists"]["far_hf"]
    del fh
    assert O.records_digest(fl) == m["lists"]["far_lf"]


@pytest.mark.gpu
def test_sphere2m_device_walk_is_bit_exact(gpu):
    m = meta()
    D = build(True, False)
    assert D.info("plan_walk_device") == 1 and D.info("tree_device") == 1
    check_counts(D, m)
    for tag in "TS":
        assert digest(*D.tree(tag)) == m[f"tree_{tag}"], tag
    dptr, dsrc, dtab = D.m2l_entries()
    dnear = D.near_digest()
    del D
    H = build(False, False)
    assert H.info("plan_walk_device") == 0
    # near-field chunks, symmetric blocks, reduction rows and work items
    assert np.array_equal(dnear, H.near_digest())
    hptr, hsrc, htab = H.m2l_entries()
    assert np.array_equal(dptr, hptr)
    assert np.array_equal(dsrc, hsrc)
    assert np.array_equal(dtab, htab)
