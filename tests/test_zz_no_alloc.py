"""defmm_direct_noalloc through the C ABI: direct sums whose scratch is a
fixed device array of the library, checked against defmm_check_full (the
same FP64 direct sums with allocated scratch) and the oracle.

Collected last on purpose: it must also pass after every other test of the
session has used the device (and alone, in a fresh process).
"""
import numpy as np
import pytest

from defmm_b200 import IBFMM_Mat, DefmmError
from oracle import oracle as O
from tests.golden.cases import case_inputs

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-12
MAX_TARGETS = 262144
M64 = (1 << 64) - 1


def check_full_sample(nt, nsamples, seed):
    """The target indices defmm_check_full samples: seeded partial
    Fisher-Yates with splitmix64, then sorted."""
    idx = list(range(nt))
    s = seed
    for i in range(min(nsamples, nt)):
        s = (s + 0x9E3779B97F4A7C15) & M64
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        z ^= z >> 31
        j = i + z % (nt - i)
        idx[i], idx[j] = idx[j], idx[i]
    return np.sort(np.array(idx[:min(nsamples, nt)], dtype=np.int64))


def norms(ex, fm):
    d, m = np.abs(ex - fm), np.abs(ex)
    return np.array([d.max() / m.max(), d.sum() / m.sum(), np.sqrt((d * d).sum() / (m * m).sum())])


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_direct_noalloc_matches_check_full(gpu):
    import torch
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube20k")
    A = IBFMM_Mat()
    A.addSourceParticles(src)
    A.addTargetParticles(trg)
    A.prcmpt(L, ncrit, kappa, lvmax)
    p = A.matvec(q)
    runs = [(300, 3), (2000, 11)]
    ref = [A.check_full(n, seed) for n, seed in runs]
    idx = [check_full_sample(len(trg), n, seed) for n, seed in runs]
    d_t = [torch.from_numpy(np.ascontiguousarray(trg[i])).cuda() for i in idx]
    d_o = [torch.empty(len(i), dtype=torch.complex128, device="cuda") for i in idx]
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    # two calls in a row on one stream, sharing the library's scratch
    for k in range(2):
        A.direct_noalloc(d_t[k].data_ptr(), len(idx[k]), d_o[k].data_ptr(), stream)
    torch.cuda.synchronize()
    for k in range(2):
        ex = d_o[k].cpu().numpy()
        assert rel(ex, O.direct(src, q, trg[idx[k]], kappa)) <= FP64_TOL
        # the norms are relative errors: direct sums that agree to a relative
        # delta move them by at most delta * (1 + norm)
        e = norms(ex, p[idx[k]])
        e_ref = np.array([ref[k]["linf"], ref[k]["l1"], ref[k]["l2"]])
        assert np.all(np.abs(e - e_ref) <= FP64_TOL * (1 + e_ref))


def test_direct_noalloc_allocates_nothing_and_fills_the_scratch(gpu):
    """After one warm-up call (which may load the library's device image),
    further calls leave the device's free memory unchanged; a call with the
    maximum 262,144 targets (the scratch holds one source chunk then) agrees
    with the oracle's FP64 direct sums on a subsample."""
    import torch
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_lf")
    A = IBFMM_Mat()
    A.addSourceParticles(src)
    A.addTargetParticles(trg)
    A.prcmpt(L, ncrit, kappa, lvmax)
    A.matvec(q)
    reps = MAX_TARGETS // len(trg) + 1
    big = np.ascontiguousarray(np.tile(trg, (reps, 1))[:MAX_TARGETS])
    d_t = torch.from_numpy(big).cuda()
    d_o = torch.empty(MAX_TARGETS, dtype=torch.complex128, device="cuda")
    small = torch.from_numpy(np.ascontiguousarray(trg[:1000])).cuda()
    d_s = torch.empty(1000, dtype=torch.complex128, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    A.direct_noalloc(small.data_ptr(), 1000, d_s.data_ptr(), stream)  # warm-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        A.direct_noalloc(small.data_ptr(), 1000, d_s.data_ptr(), stream)
        A.direct_noalloc(d_t.data_ptr(), MAX_TARGETS, d_o.data_ptr(), stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    ex = d_o.cpu().numpy()
    sub = np.sort(np.random.default_rng(3).choice(MAX_TARGETS, size=300, replace=False))
    assert rel(ex[sub], O.direct(src, q, big[sub], kappa)) <= FP64_TOL
    # a target repeated in the tiled set gets the same sum every time
    n = len(trg)
    np.testing.assert_array_equal(ex[:1000], ex[n:n + 1000])
    # the 1,000-target calls split the sources into chunks: same sums to rounding
    assert rel(d_s.cpu().numpy(), ex[:1000]) <= FP64_TOL


def test_direct_noalloc_read_finishes_before_next_host_gemv(gpu):
    """The direct sums read the handle's copy of the charges on the caller's
    stream; a host gemv with new charges issued right after, on the handle's
    own stream, must not overwrite them before that read."""
    import torch
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_lf")
    A = IBFMM_Mat()
    A.addSourceParticles(src)
    A.addTargetParticles(trg)
    A.prcmpt(L, ncrit, kappa, lvmax)
    A.matvec(q)
    d_t = torch.from_numpy(np.ascontiguousarray(np.tile(trg, (13, 1))[:MAX_TARGETS])).cuda()
    d_o = torch.empty(d_t.shape[0], dtype=torch.complex128, device="cuda")
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    A.direct_noalloc(d_t.data_ptr(), d_t.shape[0], d_o.data_ptr(), side.cuda_stream)
    A.matvec(2.0 * q)  # new charges copied on the handle's stream
    torch.cuda.synchronize()
    ex = d_o[:200].cpu().numpy()
    assert rel(ex, O.direct(src, q, trg[:200], kappa)) <= FP64_TOL


def test_direct_noalloc_rejects_more_targets_than_scratch(gpu):
    import torch
    src, trg, q, L, ncrit, kappa, lvmax = case_inputs("cube_lf")
    A = IBFMM_Mat()
    A.addSourceParticles(src)
    A.addTargetParticles(trg)
    A.prcmpt(L, ncrit, kappa, lvmax)
    A.matvec(q)
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    # rejected on the host before anything is launched
    with pytest.raises(DefmmError, match="262144"):
        A.direct_noalloc(d.data_ptr(), MAX_TARGETS + 1, d.data_ptr())
