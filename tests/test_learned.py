"""Order-selection network (defmm_b200/learned.py, csrc/mlp.cu): the CUDA
forward, backward, Adam and BF16 inference kernels against the numpy oracle
(oracle/mlp_ref.py); the oracle's gradient against finite differences; the
committed network on the held-out problems of the committed order sweep,
and one matvec at a chosen order checked by FP64 direct sums."""
import ctypes
import math
import os

import numpy as np
import pytest

from defmm_b200 import learned as Lr
from oracle import mlp_ref as R


def rand_params(seed):
    rng = np.random.default_rng(seed)
    return (0.3 * rng.standard_normal(R.NPARAM)).astype(np.float32)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rand_params(1).astype(np.float64)
    X = rng.standard_normal((20, R.NIN))
    y = rng.integers(0, R.NOUT, 20)
    w = rng.uniform(0.5, 2.0, 20)
    _, g = R.loss_and_grad(p, X, y, w)
    for k in rng.choice(R.NPARAM, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (R.loss_and_grad(pp, X, y, w)[0] - R.loss_and_grad(pm, X, y, w)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd)


def test_parameter_layout_matches_header():
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "defmm_b200.h")).read()
    assert f"#define DEFMM_MLP_PARAMS {R.NPARAM}" in hdr
    assert R.NPARAM == Lr.NPARAM == Lr.init_params().size


def test_labels_pick_the_lowest_order_meeting_the_tolerance():
    err = np.array([[1e-2, 3e-3, 4e-4, 5e-5, 1e-5, 3e-6]])
    y, ok = Lr.labels(err, tols=np.array([5e-2, 1e-3, 1e-5, 1e-7]))
    assert list(y) == [0, 2, 4, 5] and list(ok) == [True, True, True, False]
    y2, _ = Lr.labels(err, tols=np.array([1e-3]), margin=4.0)  # 4 x 4e-4 > 1e-3
    assert list(y2) == [3]


def test_held_out_split_covers_every_kind():
    d = np.load(Lr.SWEEP_PATH)
    tr, te = Lr.split(len(d["err"]))
    assert set(d["kind"][te]) == set(d["kind"][tr]) == {"cube", "sphere", "blobs", "spheroid", "mixture"}


def test_features_are_deterministic_and_finite():
    rng1, rng2 = np.random.default_rng(5), np.random.default_rng(5)
    for i in range(5):
        a = Lr.sample_problem(rng1, i)
        b = Lr.sample_problem(rng2, i)
        fa = Lr.features(a[1], a[2], a[3], 1e-4)
        assert np.array_equal(fa, Lr.features(b[1], b[2], b[3], 1e-4))
        assert fa.shape == (Lr.NIN,) and np.all(np.isfinite(fa))


def test_committed_sweep_features_regenerate_from_the_seed():
    # the sweep's inputs come from the seeded problem generator: replaying
    # it reproduces the recorded features of the first problems exactly
    d = np.load(Lr.SWEEP_PATH)
    rng = np.random.default_rng(int(d["seed"]))
    for i in range(4):
        kind, pts, kappa, ncrit = Lr.sample_problem(rng, i)
        assert kind == d["kind"][i] and len(pts) == d["n"][i]
        assert np.array_equal(Lr.problem_features(pts, kappa, ncrit), d["feat"][i])


def test_committed_sweep_and_model_load():
    d = np.load(Lr.SWEEP_PATH)
    assert d["feat"].shape[1] == Lr.NIN - 1 and d["err"].shape[1] == len(Lr.ORDERS)
    m = Lr.OrderModel.load()
    assert m.params.shape == (Lr.NPARAM,) and np.all(np.isfinite(m.params))


# ---------------------------------------------------------------- GPU parts
def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.gpu
def test_kernels_match_oracle(gpu):
    import torch
    from defmm_b200.api import lib
    rng = np.random.default_rng(3)
    n = 300
    p = rand_params(2)
    X = rng.standard_normal((n, R.NIN)).astype(np.float32)
    y = rng.integers(0, R.NOUT, n).astype(np.int32)
    w = rng.uniform(0.5, 2.0, n).astype(np.float32)
    dp, dX, dy, dw = _dev(p), _dev(X), _dev(y), _dev(w)
    H1 = torch.empty((n, R.NH), dtype=torch.float32, device="cuda")
    H2, Z = torch.empty_like(H1), torch.empty((n, R.NOUT), dtype=torch.float32, device="cuda")
    g = torch.zeros(R.NPARAM, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    scr = torch.empty(n * (R.NOUT + 2 * R.NH), dtype=torch.float32, device="cuda")
    L = lib()
    assert L.defmm_mlp_forward(dp.data_ptr(), dX.data_ptr(), n, H1.data_ptr(), H2.data_ptr(), Z.data_ptr(),
                               None) == 0
    assert L.defmm_mlp_backward(dp.data_ptr(), dX.data_ptr(), H1.data_ptr(), H2.data_ptr(), Z.data_ptr(),
                                dy.data_ptr(), dw.data_ptr(), ctypes.c_float(float(w.sum())), n, g.data_ptr(),
                                loss.data_ptr(), scr.data_ptr(), None) == 0
    torch.cuda.synchronize()
    _, _, z = R.forward(p, X)
    assert np.max(np.abs(Z.cpu().numpy() - z)) <= 1e-4 * (1 + np.max(np.abs(z)))
    ref_loss, ref_g = R.loss_and_grad(p, X, y, w)
    assert abs(float(loss.item()) - ref_loss) <= 1e-5 * (1 + ref_loss)
    assert np.linalg.norm(g.cpu().numpy() - ref_g) <= 1e-4 * np.linalg.norm(ref_g)
    # one Adam step from zero moments, with weight decay
    m, v = torch.zeros_like(g), torch.zeros_like(g)
    assert L.defmm_mlp_adam(dp.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), 1, ctypes.c_float(1e-3),
                            ctypes.c_float(1e-2), None) == 0
    torch.cuda.synchronize()
    ref_p, _, _ = R.adam(p.astype(np.float64), g.cpu().numpy().astype(np.float64), 0.0, 0.0, 1, 1e-3, 1e-2)
    assert np.max(np.abs(dp.cpu().numpy() - ref_p)) <= 1e-6


@pytest.mark.gpu
def test_bf16_inference_matches_bf16_oracle(gpu):
    import torch
    from defmm_b200.api import lib
    rng = np.random.default_rng(4)
    n = 257
    p = rand_params(5)
    X = rng.standard_normal((n, R.NIN)).astype(np.float32)
    dp, dX = _dev(p), _dev(X)
    pb = torch.empty(R.NPARAM, dtype=torch.int16, device="cuda")
    out = torch.empty((n, R.NOUT), dtype=torch.float32, device="cuda")
    assert lib().defmm_mlp_to_bf16(dp.data_ptr(), pb.data_ptr(), None) == 0
    assert lib().defmm_mlp_infer_bf16(pb.data_ptr(), dX.data_ptr(), n, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(pb.cpu().numpy().view(np.uint16),
                          (R.bf16_round(p).view(np.uint32) >> 16).astype(np.uint16))
    _, _, zb = R.forward(R.bf16_round(p).astype(np.float64), X)   # BF16 weights, exact arithmetic
    _, _, z = R.forward(p.astype(np.float64), X)
    got = out.cpu().numpy()
    assert np.max(np.abs(got - zb)) <= 1e-4 * (1 + np.max(np.abs(zb)))
    assert np.max(np.abs(got - z)) <= 0.05 * (1 + np.max(np.abs(z)))   # BF16 rounding of the weights


@pytest.mark.gpu
def test_training_fits_a_separable_problem(gpu):
    rng = np.random.default_rng(6)
    X = rng.standard_normal((600, R.NIN))
    y = np.digitize(X[:, 0] + 0.5 * X[:, 1], [-1.5, -0.5, 0.0, 0.5, 1.5]).astype(np.int32)
    m = Lr.train(X, y, steps=400, lr=1e-2, wd=0.0, log_every=0)
    pred = np.argmax(m.logits(X), axis=1)
    assert np.mean(pred == y) >= 0.9


def held_out_choices(m, d, tols):
    _, test = Lr.split(len(d["err"]))
    cases = [(i, t) for i in test for t in tols]
    z = m.logits(np.array([np.append(d["feat"][i], math.log10(t)) for i, t in cases]))
    pr = np.exp(z - z.max(axis=1, keepdims=True))
    pr /= pr.sum(axis=1, keepdims=True)
    out = []
    for r, (i, t) in enumerate(cases):
        ok = np.nonzero(np.cumsum(pr[r]) >= 0.9)[0]
        learned = len(ok) > 0 and ok[0] < len(Lr.ORDERS) - 1
        out.append((i, t, Lr.ORDERS[ok[0]] if learned else 6, learned))
    return out


@pytest.mark.gpu
def test_committed_network_on_held_out_problems(gpu):
    """Held-out problems of the committed sweep (every geometry kind),
    tolerances 1e-2..1e-4, which the fixed order 6 always meets: the chosen
    orders (BF16 inference) meet every tolerance in the recorded FP64
    direct-sum errors and cost less time than order 6."""
    d = np.load(Lr.SWEEP_PATH)
    m = Lr.OrderModel.load()
    met = fixed_met = total = 0
    t_learned = t_fixed = 0.0
    k6 = Lr.ORDERS.index(6)
    for i, tol, order, _ in held_out_choices(m, d, (1e-2, 1e-3, 1e-4)):
        k = Lr.ORDERS.index(order)
        total += 1
        met += d["err"][i][k] <= tol
        fixed_met += d["err"][i][k6] <= tol
        t_learned += d["ms_mixed"][i][k]
        t_fixed += d["ms_mixed"][i][k6]
    assert met == total and fixed_met == total
    assert t_learned < 0.8 * t_fixed


@pytest.mark.gpu
def test_committed_network_beats_the_fixed_order_at_tight_tolerances(gpu):
    """At 1e-6 the fixed order 6 misses on almost every held-out problem.
    Where the network is confident its order meets the tolerance (>= 90% of
    those cases), elsewhere it falls back to order 6; overall it meets the
    tolerance more often than the fixed order."""
    d = np.load(Lr.SWEEP_PATH)
    m = Lr.OrderModel.load()
    k6 = Lr.ORDERS.index(6)
    ch = held_out_choices(m, d, (1e-6,))
    conf = [(i, t, o) for i, t, o, learned in ch if learned]
    met_conf = sum(d["err"][i][Lr.ORDERS.index(o)] <= t for i, t, o in conf)
    met = sum(d["err"][i][Lr.ORDERS.index(o)] <= t for i, t, o, _ in ch)
    fixed = sum(d["err"][i][k6] <= t for i, t, _, _ in ch)
    assert len(conf) > 0 and met_conf >= 0.9 * len(conf)
    assert met > fixed


@pytest.mark.gpu
def test_chosen_order_is_checked_by_direct_sums(gpu):
    """One fresh problem (not in the sweep): the network's order for 1e-3,
    run and checked against FP64 direct sums at 2,000 targets."""
    from defmm_b200 import IBFMM_Mat, workloads as W
    m = Lr.OrderModel.load()
    w = W.sphere_surface(60_000, seed=99, wavelengths=12.0)
    order, learned = m.choose(w.points, w.kappa, 64, 1e-3)
    A = IBFMM_Mat()
    A.addSourceParticles(w.points)
    A.addTargetParticles(w.points)
    A.prcmpt(order, 64, w.kappa)
    A.matvec(W.charges(w.n, 3))
    err = A.check_full(2000, seed=7)["l2"]
    assert learned and order < 6 and err <= 1e-3
