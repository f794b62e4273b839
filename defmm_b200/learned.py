"""Learned order selection: a small network that predicts the lowest
interpolation order (3..8) whose matvec meets a requested relative accuracy
against FP64 direct sums, from features of the problem.

The operator uses one interpolation order for the whole tree, so the network
decides per problem (not per cell): the order is its output and the
requested tolerance one of its inputs beside the geometry.  Everything the
network learns from is generated by the method itself: ``generate`` sweeps
orders 3..8 on seeded synthetic problems and records the relative L2 error
of the FP64 matvec against FP64 direct sums at 2,000 seeded targets
(``defmm_check_full``) and the matvec times.  ``train`` fits the network on
the GPU with the library's own kernels (``defmm_mlp_*``: FP32 forward,
backward and Adam); ``OrderModel.choose`` runs the BF16 inference kernel and
falls back to the fixed order whenever the predicted probability of meeting
the tolerance is below ``confidence`` at every order below 8.  Every matvec
run at a chosen order can be checked by ``defmm_check_full``.

    python -m defmm_b200.learned generate --out sweep.npz --problems 300
    python -m defmm_b200.learned train --data sweep.npz --out order_mlp.npz

The committed sweep and network are defmm_b200/data/order_sweep.npz and
defmm_b200/data/order_mlp.npz.
"""
from __future__ import annotations

import argparse
import ctypes
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from . import workloads as W
from .api import DefmmError, IBFMM_Mat, lib

ORDERS = (3, 4, 5, 6, 7, 8)
NIN, NH, NOUT, NPARAM = 12, 64, 6, 5382
FEATURES = ("log10_n", "log2_wavelengths", "log10_pts_per_wl2", "dimension", "log10_pts_per_cell",
            "extent_mid", "extent_min", "pca_flatness", "leaf_size", "kappa_leaf", "clustering", "log10_tol")
DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
SWEEP_PATH = os.path.join(DATA, "order_sweep.npz")
MODEL_PATH = os.path.join(DATA, "order_mlp.npz")


# ------------------------------------------------------------------ features
def problem_features(points: np.ndarray, kappa: float, ncrit: int) -> np.ndarray:
    """The 11 geometry features (all but the tolerance), float64:
    log10 N; log2 of the wavelengths across the bounding-box diagonal; log10
    points per square wavelength of the occupied surface measure; occupied-
    cell dimension log2(cells at 32^3 / cells at 16^3) (2 for surfaces, 3 for
    volumes); log10 points per occupied 32^3 cell; middle and smallest box
    extent over the largest; covariance flatness (smallest / largest
    eigenvalue); leaf size / 64; k times the estimated leaf diameter; the
    fraction of points in the densest 1% of occupied cells."""
    P = np.asarray(points, dtype=np.float64)
    n = P.shape[0]
    lo, hi = P.min(axis=0), P.max(axis=0)
    ext = hi - lo
    side = max(float(ext.max()), 1e-300)
    diag = float(np.linalg.norm(ext))
    wl = 2.0 * math.pi / kappa if kappa > 0 else math.inf

    def occupied(g):
        idx = np.clip(np.floor((P - lo) / side * g), 0, g - 1).astype(np.int64)
        keys = (idx[:, 0] * g + idx[:, 1]) * g + idx[:, 2]
        return np.unique(keys, return_counts=True)[1]

    c16, c32 = occupied(16), occupied(32)
    dim = math.log2(len(c32) / len(c16))
    cell = side / 32.0
    measure = len(c32) * cell ** 2  # surface-measure proxy of the occupied cells
    pts_wl2 = n / max(measure / wl ** 2, 1e-300) if math.isfinite(wl) else float(n)
    e = np.sort(ext) / side
    ev = np.sort(np.linalg.eigvalsh(np.cov(P.T)))
    leaf = side * (ncrit / n) ** (1.0 / max(dim, 1.0))
    top = np.sort(c32)[::-1]
    k = max(1, len(top) // 100)
    return np.array([
        math.log10(n),
        math.log2(max(kappa * diag / (2.0 * math.pi), 1e-3)),
        math.log10(max(pts_wl2, 1e-3)),
        dim,
        math.log10(n / len(c32)),
        e[1], e[0],
        ev[0] / max(ev[-1], 1e-300),
        ncrit / 64.0,
        kappa * leaf * math.sqrt(3.0),
        float(top[:k].sum()) / n,
    ])


def features(points, kappa, ncrit, tol) -> np.ndarray:
    return np.append(problem_features(points, kappa, ncrit), math.log10(tol))


# ------------------------------------------------------------------ problems
def sample_problem(rng: np.random.Generator, i: int):
    """Seeded synthetic problem i: geometry cycling cube surface (edge-
    refined), sphere surface, Gaussian blobs (sigma 0.01-0.1), spheroid, and
    the 40/30/30 mixture of cube surface, sphere of radius 0.4 and blobs;
    N log-uniform in [20,000, 200,000]; 2-48 wavelengths across the
    diameter, capped at sqrt(N / (25 pi)); leaf size 32, 64 or 96."""
    kind = ("cube", "sphere", "blobs", "spheroid", "mixture")[i % 5]
    n = int(round(math.exp(rng.uniform(math.log(2e4), math.log(2e5)))))
    wl = math.exp(rng.uniform(math.log(2.0), math.log(48.0)))
    wl = max(1.0, min(wl, math.sqrt(n / (25.0 * math.pi))))
    ncrit = int(rng.choice([32, 64, 96]))
    seed = int(rng.integers(1 << 30))
    if kind == "cube":
        pts = W.cube_surface(n, seed=seed).points
        kappa = 2.0 * math.pi * wl / math.sqrt(3.0)
    elif kind == "sphere":
        pts = W.sphere_surface(n, seed=seed).points
        kappa = 2.0 * math.pi * wl / 2.0
    elif kind == "blobs":
        w = W.gaussian_blobs(n, seed=seed, sigma=float(rng.uniform(0.01, 0.1)), wavelengths=wl)
        pts, kappa = w.points, w.kappa
    elif kind == "spheroid":
        w = W.spheroid(n, seed=seed, wavelengths=wl)
        pts, kappa = w.points, w.kappa
    else:
        pts = mixture(n, seed)
        kappa = 2.0 * math.pi * wl / math.sqrt(3.0)
    return kind, np.ascontiguousarray(pts), float(kappa), ncrit


def mixture(n: int, seed: int) -> np.ndarray:
    """40% cube surface, 30% sphere surface of radius 0.4, 30% Gaussian blobs
    with sigma in [0.01, 0.1], all in the unit cube."""
    rng = np.random.default_rng(seed)
    n1, n2 = int(0.4 * n), int(0.3 * n)
    n3 = n - n1 - n2
    a = W.cube_surface(n1, seed=seed + 1).points
    b = 0.4 * W.sphere_surface(n2, seed=seed + 2).points
    sig = rng.uniform(0.01, 0.1, size=8)
    centres = rng.uniform(-0.3, 0.3, size=(8, 3))
    which = rng.integers(0, 8, size=n3)
    c = np.clip(centres[which] + sig[which, None] * rng.standard_normal((n3, 3)), -0.5, 0.5)
    p = np.concatenate([a, b, c])
    return p[rng.permutation(n)]


# ---------------------------------------------------------------- generation
def sweep_problem(points, kappa, ncrit, q, orders=ORDERS, nsamples=2000):
    """At each order: relative L2 error of the FP64 matvec against FP64
    direct sums at `nsamples` seeded targets, and the device time of one FP64
    and one mixed matvec (ms)."""
    import torch
    err, ms64, ms32 = [], [], []
    dq = torch.from_numpy(q).cuda()
    dp = torch.empty(len(q), dtype=torch.complex128, device="cuda")
    stream = torch.cuda.Stream()
    for L in orders:
        A = IBFMM_Mat()
        A.addSourceParticles(points)
        A.addTargetParticles(points)
        A.prcmpt(L, ncrit, kappa)
        A.matvec(q)
        err.append(A.check_full(nsamples, seed=7)["l2"])
        for prec, out in (("fp64", ms64), ("mixed", ms32)):
            A.set_precision(prec)
            A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            A.matvec_device(dq.data_ptr(), dp.data_ptr(), 1, stream.cuda_stream)
            e1.record(stream)
            stream.synchronize()
            out.append(e0.elapsed_time(e1))
        del A
    return np.array(err), np.array(ms64), np.array(ms32)


def generate(nproblems: int, seed: int, out: str) -> None:
    rng = np.random.default_rng(seed)
    rows = {"feat": [], "err": [], "ms_fp64": [], "ms_mixed": [], "n": [], "kind": []}
    t0 = time.time()
    for i in range(nproblems):
        kind, pts, kappa, ncrit = sample_problem(rng, i)
        q = W.charges(len(pts), seed + i)
        e, m64, m32 = sweep_problem(pts, kappa, ncrit, q)
        rows["feat"].append(problem_features(pts, kappa, ncrit))
        rows["err"].append(e)
        rows["ms_fp64"].append(m64)
        rows["ms_mixed"].append(m32)
        rows["n"].append(len(pts))
        rows["kind"].append(kind)
        print(f"[{i + 1}/{nproblems}] {kind} n={len(pts)} err={np.array2string(e, precision=2)} "
              f"({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(out, **{k: np.array(v) for k, v in rows.items()}, orders=np.array(ORDERS), seed=seed)


# ------------------------------------------------------------------ training
TOLS_TRAIN = np.logspace(-1.5, -7.0, 23)


def labels(err: np.ndarray, tols=TOLS_TRAIN, margin: float = 1.0):
    """Per (problem, tolerance): index of the lowest order with
    margin * error <= tol, or the last index (order 8) with reachable =
    False.  Training uses margin 2: an order counts only when it meets the
    tolerance with a factor 2 to spare."""
    y, ok = [], []
    for e in err:
        for t in tols:
            hit = np.nonzero(margin * e <= t)[0]
            y.append(int(hit[0]) if len(hit) else len(ORDERS) - 1)
            ok.append(bool(len(hit)))
    return np.array(y, dtype=np.int32), np.array(ok)


def expand(feat: np.ndarray, err: np.ndarray, tols=TOLS_TRAIN, margin: float = 2.0):
    X = np.concatenate([np.repeat(feat, len(tols), axis=0),
                        np.tile(np.log10(tols), len(feat))[:, None]], axis=1)
    y, ok = labels(err, tols, margin)
    return X.astype(np.float64), y, ok


@dataclass
class OrderModel:
    params: np.ndarray  # float32, NPARAM
    mean: np.ndarray    # feature normalisation
    std: np.ndarray

    def save(self, path: str) -> None:
        np.savez(path, params=self.params, mean=self.mean, std=self.std, features=np.array(FEATURES),
                 orders=np.array(ORDERS))

    @staticmethod
    def load(path: str = MODEL_PATH) -> "OrderModel":
        d = np.load(path)
        return OrderModel(d["params"].astype(np.float32), d["mean"], d["std"])

    def normalise(self, X: np.ndarray) -> np.ndarray:
        return ((np.asarray(X, dtype=np.float64) - self.mean) / self.std).astype(np.float32)

    def logits(self, X: np.ndarray) -> np.ndarray:
        """BF16 inference on the GPU (defmm_mlp_infer_bf16)."""
        import torch
        Xn = torch.from_numpy(self.normalise(np.atleast_2d(X))).cuda()
        p = torch.from_numpy(self.params).cuda()
        pb = torch.empty(NPARAM, dtype=torch.int16, device="cuda")
        out = torch.empty((Xn.shape[0], NOUT), dtype=torch.float32, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        _check(lib().defmm_mlp_to_bf16(p.data_ptr(), pb.data_ptr(), s))
        _check(lib().defmm_mlp_infer_bf16(pb.data_ptr(), Xn.data_ptr(), Xn.shape[0], out.data_ptr(), s))
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def choose(self, points, kappa, ncrit, tol, fixed_order=6, confidence=0.9):
        """(order, learned): the lowest order whose predicted probability of
        meeting `tol` (the cumulative probability of the classes up to it) is
        at least `confidence`; the fixed order when only order 8 qualifies."""
        z = self.logits(features(points, kappa, ncrit, tol)[None, :])[0]
        pr = np.exp(z - z.max())
        pr /= pr.sum()
        ok = np.nonzero(np.cumsum(pr) >= confidence)[0]
        if len(ok) == 0 or ok[0] == len(ORDERS) - 1:
            return fixed_order, False
        return ORDERS[int(ok[0])], True


def _check(st):
    if st != 0:
        raise DefmmError(st, "order-selection network kernel failed")


def train(X: np.ndarray, y: np.ndarray, wts=None, steps: int = 2000, lr: float = 3e-3, wd: float = 1e-3,
          seed: int = 0, log_every: int = 500) -> OrderModel:
    """Full-batch Adam with decoupled weight decay on the GPU with
    defmm_mlp_forward/backward/adam."""
    import torch
    mean, std = X.mean(axis=0), X.std(axis=0) + 1e-9
    model = OrderModel(init_params(seed), mean, std)
    n = X.shape[0]
    dev = "cuda"
    Xd = torch.from_numpy(model.normalise(X)).to(dev)
    yd = torch.from_numpy(np.asarray(y, dtype=np.int32)).to(dev)
    w = np.ones(n, dtype=np.float32) if wts is None else np.asarray(wts, dtype=np.float32)
    wt = torch.from_numpy(w).to(dev)
    p = torch.from_numpy(model.params.copy()).to(dev)
    g = torch.zeros(NPARAM, dtype=torch.float32, device=dev)
    m = torch.zeros_like(g)
    v = torch.zeros_like(g)
    H1 = torch.empty((n, NH), dtype=torch.float32, device=dev)
    H2 = torch.empty_like(H1)
    Z = torch.empty((n, NOUT), dtype=torch.float32, device=dev)
    scr = torch.empty(n * (NOUT + 2 * NH), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    L = lib()
    for it in range(1, steps + 1):
        _check(L.defmm_mlp_forward(p.data_ptr(), Xd.data_ptr(), n, H1.data_ptr(), H2.data_ptr(), Z.data_ptr(), s))
        _check(L.defmm_mlp_backward(p.data_ptr(), Xd.data_ptr(), H1.data_ptr(), H2.data_ptr(), Z.data_ptr(),
                                    yd.data_ptr(), wt.data_ptr(), ctypes.c_float(float(w.sum())), n, g.data_ptr(),
                                    loss.data_ptr(), scr.data_ptr(), s))
        _check(L.defmm_mlp_adam(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), it, ctypes.c_float(lr),
                                ctypes.c_float(wd), s))
        if log_every and it % log_every == 0:
            print(f"step {it}: loss {float(loss.item()):.4f}", flush=True)
    torch.cuda.synchronize()
    model.params = p.cpu().numpy()
    return model


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((NIN, NH), (NH, NH), (NH, NOUT)):
        b = math.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-b, b, size=fan_out * fan_in))
        parts.append(np.zeros(fan_out))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == NPARAM
    return p


def split(nprob: int, test_every: int = 7):
    """Problem indices of the training and held-out sets: every 7th problem
    (offset 3) is held out; 7 is prime to the 5 geometry kinds, so every kind
    is in both sets."""
    idx = np.arange(nprob)
    test = idx[idx % test_every == 3]
    return np.setdiff1d(idx, test), test


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m defmm_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("generate")
    g.add_argument("--problems", type=int, default=300)
    g.add_argument("--seed", type=int, default=2024)
    g.add_argument("--out", default=SWEEP_PATH)
    t = sub.add_parser("train")
    t.add_argument("--data", default=SWEEP_PATH)
    t.add_argument("--out", default=MODEL_PATH)
    t.add_argument("--steps", type=int, default=2000)
    a = ap.parse_args(argv)
    if a.cmd == "generate":
        generate(a.problems, a.seed, a.out)
    else:
        d = np.load(a.data)
        tr, _ = split(len(d["err"]))
        X, y, _ = expand(d["feat"][tr], d["err"][tr])
        train(X, y, steps=a.steps).save(a.out)


if __name__ == "__main__":
    main()
