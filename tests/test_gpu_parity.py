"""GPU parity: the CUDA matvec through the C ABI against the oracle (the
C++ restatement, itself pinned to the reference by tests/test_oracle.py) and
against the reference's golden samples.

Tolerances: plain FP64 path <= 1e-12 relative L2 (the reference's own
summation order differs, so bitwise equality is not expected); mixed
precision <= 1e-6 relative L2 against the FP64 path.
"""
import json
import os

import numpy as np
import pytest

from defmm_b200 import IBFMM_Mat, workloads as W
from oracle import oracle as O
from tests.golden.cases import CASES, case_inputs
from tests.golden.gen_golden import sample_index

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FP64_TOL = 1e-12
MIXED_TOL = 1e-6


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def make(src, trg, L, ncrit, kappa, lvmax=-1):
    A = IBFMM_Mat()
    A.addSourceParticles(src)
    A.addTargetParticles(trg)
    A.prcmpt(L, ncrit, kappa, lvmax)
    return A


@pytest.mark.parametrize("name", CASES)
def test_fp64_matches_oracle_and_reference_samples(name, gpu):
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    A = make(src, trg, L, ncrit, kappa, lvmax)
    p = A.matvec(q)
    po = O.OracleFMM(src, trg, L, ncrit, kappa, lvmax).gemv(q)
    assert rel(p, po) <= FP64_TOL
    sample = np.load(os.path.join(GOLD, f"{name}_pot_sample.npy"))
    assert rel(p[sample_index(trg.shape[0])], sample) <= FP64_TOL


@pytest.mark.parametrize("order", [2, 3, 7, 8])
def test_orders_outside_the_golden_cases_match_oracle(order, gpu):
    # the golden cases run orders 4-6; the order-selection network also picks
    # 3, 7 and 8, and the kernels are instantiated for 2-8
    w = W.sphere_surface(8000, seed=21, wavelengths=6.0)
    q = W.charges(w.n, 4)
    A = make(w.points, w.points, order, 64, w.kappa)
    p = A.matvec(q)
    assert rel(p, O.OracleFMM(w.points, w.points, order, 64, w.kappa, -1).gemv(q)) <= FP64_TOL
    A.set_precision("mixed")
    assert rel(A.matvec(q), p) <= MIXED_TOL


@pytest.mark.parametrize("name", ["cube20k", "cube_lf", "blobs_sphere", "cube_laplace"])
def test_mixed_matches_fp64(name, gpu):
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    A = make(src, trg, L, ncrit, kappa, lvmax)
    p64 = A.matvec(q)
    A.set_precision("mixed")
    p32 = A.matvec(q)
    assert rel(p32, p64) <= MIXED_TOL


def test_repeated_gemv_is_correct_every_time(gpu):
    # the reference's gemv is only valid on its first call after prcmpt
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_lf")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    p1 = A.matvec(q)
    p2 = A.matvec(q)
    assert np.array_equal(p1, p2)
    p3 = A.matvec(2 * q)
    assert rel(p3, 2 * p1) <= 1e-14


def test_batched_rhs_equal_single(gpu):
    # several host right-hand sides run as one block of the grouped layout;
    # each agrees with its own single-RHS matvec (resident layout) to
    # rounding: the two layouts sum the same terms in different orders
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("blobs_sphere")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    Q = np.stack([q, W.charges(len(q), 9), W.charges(len(q), 10)])
    P = A.matvec(Q)
    assert A.info("layout") == 2 and A.info("rhs_block") == 3
    for r in range(3):
        assert rel(P[r], A.matvec(Q[r])) <= 1e-13
    assert A.info("layout") == 1


def test_device_pointer_path_matches_host_path(gpu):
    import torch
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_lf")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    ph = A.matvec(q)
    dq = torch.from_numpy(q).cuda()
    dp = torch.empty(len(trg), dtype=torch.complex128, device="cuda")
    A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(dp.cpu().numpy(), ph)


def test_check_full_samples_direct_sum(gpu):
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube20k")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    p = A.matvec(q)
    e = A.check_full(300, seed=3)
    # order-4 interpolation: the reference's own error is ~6e-4 here
    assert 1e-6 < e["l2"] < 3e-3
    idx = np.sort(np.random.default_rng(0).choice(len(trg), 50, replace=False))
    ex = O.direct(src, q, trg[idx], kappa)
    assert rel(p[idx], ex) < 3e-3


def test_linearity_and_accuracy_at_larger_size(gpu):
    # size-independent properties where the oracle would take minutes
    w = W.sphere_surface(300_000, seed=5, wavelengths=48)
    A = make(w.points, w.points, 5, 64, w.kappa)
    q1, q2 = W.charges(w.n, 1), W.charges(w.n, 2)
    p1, p2 = A.matvec(q1), A.matvec(q2)
    p12 = A.matvec(q1 + 2j * q2)
    assert rel(p12, p1 + 2j * p2) <= 1e-13
    e = A.check_full(200, seed=1)
    assert e["l2"] < 1e-3
    A.set_precision("mixed")
    assert rel(A.matvec(q1), p1) <= MIXED_TOL


def test_sources_and_targets_apart(gpu):
    src = W.sphere_surface(20000, seed=3, wavelengths=8).points * 0.4
    trg = W.cube_surface(15000, seed=6).points
    q = W.charges(len(src), 4)
    A = make(src, trg, 4, 48, 2 * np.pi * 8)
    po = O.OracleFMM(src, trg, 4, 48, 2 * np.pi * 8).gemv(q)
    assert rel(A.matvec(q), po) <= FP64_TOL


def test_graph_replay_equals_direct_launches(gpu):
    # repeated matvecs replay a captured CUDA graph; results must not change
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_lf")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    A.set_graphs(False)
    p_direct = A.matvec(q)
    A.set_graphs(True)
    p1 = A.matvec(q)  # captures
    p2 = A.matvec(q)  # replays
    q2 = W.charges(len(q), 77)
    p3 = A.matvec(q2)  # replays with new input data in the same buffers
    assert np.array_equal(p1, p_direct) and np.array_equal(p2, p_direct)
    A.set_graphs(False)
    assert np.array_equal(p3, A.matvec(q2))


def test_laplace_kernel_is_the_zero_wavenumber_operator(gpu):
    # thetis_kernels.hpp:35: Laplace(R) = 1 / (4 pi R), the Helmholtz kernel
    # at k = 0; every level is low-frequency.  Against explicit 1/(4 pi r) sums.
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_laplace")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    assert A.info("cpt") == 0 and A.info("far_hf") == 0
    p = A.matvec(q)
    idx = np.sort(np.random.default_rng(1).choice(len(trg), 200, replace=False))
    d = trg[idx][:, None, :] - src[None, :, :]
    r2 = (d * d).sum(-1)
    G = np.where(r2 < 1e-16, 0.0, 1.0 / (4 * np.pi * np.sqrt(np.where(r2 < 1e-16, 1.0, r2))))
    ex = G @ q
    assert rel(p[idx], ex) < 2e-3  # order-4 interpolation error


def test_batch_of_operators_equals_individual_matvecs(gpu):
    # independent problems (different geometries, orders, wavenumbers and
    # precisions) run by one graph launch: each result is its own matvec's
    import torch
    from defmm_b200 import Batch
    ops, ins, outs, ref = [], [], [], []
    for name, prec in (("cube20k", "fp64"), ("blobs_sphere", "mixed"), ("cube_laplace", "fp64")):
        src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
        A = make(src, trg, L, ncrit, kappa, lvmax)
        A.set_precision(prec)
        ref.append(A.matvec(q))
        ops.append(A)
        ins.append(torch.from_numpy(q).cuda())
        outs.append(torch.zeros(len(trg), dtype=torch.complex128, device="cuda"))
    for lanes in (1, 2, 3):
        b = Batch(ops, [t.data_ptr() for t in ins], [t.data_ptr() for t in outs], lanes)
        for t in outs:
            t.zero_()
        torch.cuda.synchronize()
        b.launch(torch.cuda.current_stream().cuda_stream)
        b.launch(torch.cuda.current_stream().cuda_stream)  # replays give the same results
        torch.cuda.synchronize()
        for r, t in zip(ref, outs):
            assert np.array_equal(t.cpu().numpy(), r)
        del b


def test_device_multi_rhs_equals_single_calls(gpu):
    # several device right-hand sides in one call: one pass of the grouped
    # layout, against single calls on the resident layout
    import torch
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube20k")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    rng = np.random.default_rng(11)
    Q = (rng.uniform(-1, 1, (3, len(src))) + 1j * rng.uniform(-1, 1, (3, len(src)))).astype(np.complex128)
    for prec in ("fp64", "mixed"):
        A.set_precision("fp64")
        ref = [A.matvec(Q[r]) for r in range(3)]
        A.set_precision(prec)
        d_in = torch.from_numpy(Q).cuda()
        d_out = torch.zeros((3, len(trg)), dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        A.matvec_device(d_in.data_ptr(), d_out.data_ptr(), 3, 0)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        for r in range(3):
            assert rel(got[r], ref[r]) <= (1e-13 if prec == "fp64" else MIXED_TOL)


@pytest.mark.parametrize("name", CASES)
def test_grouped_layout_matches_oracle(name, gpu):
    # the direction-streamed layout (HF levels in direction groups, one
    # group's expansions at a time, LF levels resident) forced for a single
    # right-hand side: FP64 against the oracle, mixed against FP64
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    A = make(src, trg, L, ncrit, kappa, lvmax)
    po = O.OracleFMM(src, trg, L, ncrit, kappa, lvmax).gemv(q)
    for groups in (1, 3):
        A.set_blocking(16, groups)
        A.set_precision("fp64")
        p = A.matvec(q)
        assert A.info("layout") == 2
        assert rel(p, po) <= FP64_TOL
        A.set_precision("mixed")
        assert rel(A.matvec(q), p) <= MIXED_TOL


@pytest.mark.parametrize("name", ["sphere_l6", "cube20k"])
def test_rhs_blocks_do_not_change_any_right_hand_side(name, gpu):
    # with the same direction groups, every right-hand side gets the same
    # bits whatever the block size of the pass (1, 2 or 4 of 5 vectors; the
    # last block partly filled) and however many share an M2L CTA (at order
    # 5 the inverse DFTs of a CTA's right-hand sides run as one transform);
    # the near-field, M2L and transfer arithmetic of one right-hand side does
    # not depend on its neighbours
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    A = make(src, trg, L, ncrit, kappa, lvmax)
    rng = np.random.default_rng(5)
    Q = (rng.uniform(-1, 1, (5, len(src))) + 1j * rng.uniform(-1, 1, (5, len(src)))).astype(np.complex128)
    for prec in ("fp64", "mixed"):
        A.set_precision(prec)
        A.set_blocking(1, 4)
        ref = np.stack([A.matvec(Q[r]) for r in range(5)])
        assert A.info("groups") >= (3 if name == "sphere_l6" else 1)
        for rb in (2, 4):
            for per_cta in (1, 2, 4, 8):
                A.set_blocking(rb, 4)
                A.set_rhs_per_cta(per_cta)
                P = A.matvec(Q)
                assert A.info("rhs_block") == rb
                assert np.array_equal(P, ref)
        po = O.OracleFMM(src, trg, L, ncrit, kappa, lvmax).gemv(Q[4])
        assert rel(ref[4], po) <= (FP64_TOL if prec == "fp64" else MIXED_TOL)
        A.set_blocking(16, 0)


@pytest.mark.parametrize("name", ["cube20k", "cube_lf", "blobs_sphere", "sphere_l6", "sphere_o3"])
def test_staged_m2l_matches_one_target_per_cta(name, gpu):
    # the mixed-precision M2L staged through shared memory by bulk copies
    # (four target slots per CTA over their merged lists, orders 3-6) gives
    # the bits of the one-target-slot kernel for every right-hand side, with
    # right-hand-side counts that do and do not divide its block (8, 6), and
    # with several direction groups; one right-hand side is checked against
    # the oracle
    if name == "sphere_o3":
        w = W.sphere_surface(20000, seed=12, wavelengths=8)
        src = trg = w.points
        L, ncrit, kappa, lvmax = 3, 48, w.kappa, -1
    else:
        src, trg, _, L, ncrit, kappa, lvmax = case_inputs(name)
    A = make(src, trg, L, ncrit, kappa, lvmax)
    A.set_precision("mixed")
    assert 0 < A.info("m2l_group_list") <= 2048
    rng = np.random.default_rng(7)
    for nrhs, groups in ((8, 0), (8, 3), (6, 0)):
        Q = (rng.uniform(-1, 1, (nrhs, len(src))) + 1j * rng.uniform(-1, 1, (nrhs, len(src)))).astype(np.complex128)
        A.set_blocking(nrhs, groups)
        A.set_m2l_staging(False)
        ref = A.matvec(Q)
        A.set_m2l_staging(True)
        assert A.info("m2l_staging") == 1
        P = A.matvec(Q)
        assert np.array_equal(P, ref), (nrhs, groups)
    po = O.OracleFMM(src, trg, L, ncrit, kappa, lvmax).gemv(Q[0])
    assert rel(P[0], po) <= MIXED_TOL


def small_case(name):
    if name == "sphere300":  # 3 levels, 48 far pairs
        p = W.sphere_surface(300, seed=3, wavelengths=2).points
        return p, p, 3, 32, 2 * np.pi
    if name == "cube1000":  # order 4, leaf 16
        p = W.cube_surface(1000, seed=4).points
        return p, p, 4, 16, 2 * np.pi * 4 / np.sqrt(3)
    if name == "near_only":  # a small target sphere inside source blobs: no far pair at all
        src = W.gaussian_blobs(3000, seed=5, wavelengths=4).points
        return src, W.sphere_surface(150, seed=6).points * 0.3, 4, 32, 2 * np.pi * 4 / np.sqrt(3)
    raise KeyError(name)


@pytest.mark.parametrize("name", ["sphere300", "cube1000", "near_only"])
def test_small_and_degenerate_problems(name, gpu):
    # the smallest valid trees (a few levels, tens of far pairs), and a
    # problem whose interactions are all near field: FP64 against the oracle,
    # mixed against FP64, several right-hand sides (one pass and forced
    # direction groups) against single calls
    src, trg, L, ncrit, kappa = small_case(name)
    A = make(src, trg, L, ncrit, kappa)
    rng = np.random.default_rng(11)
    Q = (rng.uniform(-1, 1, (3, len(src))) + 1j * rng.uniform(-1, 1, (3, len(src)))).astype(np.complex128)
    p = A.matvec(Q[0])
    assert rel(p, O.OracleFMM(src, trg, L, ncrit, kappa, -1).gemv(Q[0])) <= FP64_TOL
    if name == "near_only":
        assert A.info("far_hf") + A.info("far_lf") == 0
    single = np.stack([A.matvec(Q[r]) for r in range(3)])
    for groups in (0, 2):
        A.set_blocking(3, groups)
        P = A.matvec(Q)
        assert A.info("rhs_block") == 3
        for r in range(3):
            assert rel(P[r], single[r]) <= 1e-13
    A.set_precision("mixed")
    A.set_blocking(16, 0)
    assert rel(A.matvec(Q[0]), p) <= MIXED_TOL
    P = A.matvec(Q)
    for r in range(3):
        assert rel(P[r], single[r]) <= MIXED_TOL


def test_launch_choices_and_autotune_keep_results_bit_identical(gpu):
    # M2L threads per CTA, one or two target slots per M2L CTA and near-field
    # CTAs per SM change only the schedule: every combination gives the same
    # bits
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("sphere_l6")
    A = make(src, trg, L, ncrit, kappa, lvmax)
    for prec in ("fp64", "mixed"):
        A.set_precision(prec)
        ref = A.matvec(q)
        for pair in (0, 1):
            A.set_m2l_pairing(pair)
            for nt in (128, 256):
                for bps in (8, 32):
                    A.set_launch(nt, bps)
                    assert A.info("m2l_threads") == nt and A.info("p2p_blocks_per_sm") == bps
                    assert A.info("m2l_pairing") == pair
                    assert np.array_equal(A.matvec(q), ref)
        c = A.autotune(reps=1)
        assert c["m2l_threads"] in (128, 256) and c["p2p_blocks_per_sm"] in (8, 16, 32)
        assert c["m2l_pairing"] in (0, 1)
        assert A.info("m2l_threads") == c["m2l_threads"]
        sched = A.m2l_schedule()  # the autotuner's choice per level
        assert len(sched) == A.info("nlvl")
        assert all(t in (128, 256) and pr in (0, 1) for t, pr in sched)
        assert np.array_equal(A.matvec(q), ref)
        # the grouped layout runs the same per-level choices
        A.set_blocking(16, 2)
        assert np.array_equal(A.matvec(q), A.matvec(q))
        A.set_blocking(16, 0)



@pytest.mark.parametrize("order", [3, 5, 6, 7])
def test_tensor_core_p2m_matches_fp64(order, gpu):
    # P2M and L2P on the tensor cores (tcgen05, 3-pass split TF32): one M
    # tile (orders <= 5), two (6) and three (7) tiles of 128 expansion
    # entries in P2M, 4 to 11 K chunks in L2P; the sphere's leaves hold up to
    # 63 points (two K chunks of 32 in P2M)
    w = W.sphere_surface(20000, seed=23, wavelengths=8.0)
    q = W.charges(w.n, 6)
    A = make(w.points, w.points, order, 64, w.kappa)
    p64 = A.matvec(q)
    A.set_precision("mixed")
    p_cc = A.matvec(q)
    A.set_tensor_cores(True)
    p_tc = A.matvec(q)
    assert A.info("tensor_cores") == 1
    assert rel(p_tc, p64) <= MIXED_TOL
    assert rel(p_tc, p_cc) <= MIXED_TOL
    # a block of right-hand sides over the grouped layout
    rng = np.random.default_rng(8)
    Q = (rng.uniform(-1, 1, (3, w.n)) + 1j * rng.uniform(-1, 1, (3, w.n))).astype(np.complex128)
    A.set_blocking(3, 2)
    P = A.matvec(Q)
    A.set_precision("fp64")
    for r in range(3):
        assert rel(P[r], A.matvec(Q[r])) <= MIXED_TOL


@pytest.mark.parametrize("name", ["cube_lf", "blobs_sphere", "cube_laplace"])
def test_tensor_core_p2m_low_frequency_and_distinct_sets(name, gpu):
    # LF leaves (no plane-wave phases) and distinct source / target trees;
    # at order 8 the CUDA-core path stays in use
    if name == "cube_lf":
        w = W.sphere_surface(8000, seed=21, wavelengths=6.0)
        A8 = make(w.points, w.points, 8, 64, w.kappa)
        A8.set_precision("mixed")
        A8.set_tensor_cores(True)
        assert A8.info("tensor_cores") == 0
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs(name)
    A = make(src, trg, L, ncrit, kappa, lvmax)
    p64 = A.matvec(q)
    A.set_precision("mixed")
    A.set_tensor_cores(True)
    assert rel(A.matvec(q), p64) <= MIXED_TOL


def test_multifrequency_kernel_matches_direct_sums(gpu):
    # the reference's MultiFreq kernel (four wavenumbers kappa / a) as the sum
    # of four Helmholtz operators, against the FP64 direct sums of the same
    # four terms at seeded targets; the plain FP64 path against the oracle
    from defmm_b200 import MultiFreqMat
    w = W.sphere_surface(12000, seed=31, wavelengths=12.0)
    q = W.charges(w.n, 2)
    A = MultiFreqMat()
    A.addSourceParticles(w.points)
    A.addTargetParticles(w.points)
    A.prcmpt(5, 64, w.kappa)
    p = A.matvec(q)
    po = sum(O.OracleFMM(w.points, w.points, 5, 64, w.kappa / a).gemv(q) for a in A.DIVISORS)
    assert rel(p, po) <= FP64_TOL
    idx = W.sample_targets(w.n, 300, seed=3)
    ex = sum(O.direct(w.points, q, w.points[idx], w.kappa / a) for a in A.DIVISORS)
    assert rel(p[idx], ex) <= 1e-2  # the FMM's own error at order 5
    A.set_precision("mixed")
    assert rel(A.matvec(q), p) <= MIXED_TOL
