"""Python mirror of IChollet/defmm's ``IBFMM_Mat<3>`` over the C ABI of
``libdefmm_b200.so`` (include/defmm_b200.h).

Names, argument meaning and call order follow include/interface.hpp:46-224:

    A = IBFMM_Mat()
    A.addSourceParticlesINP("mesh.inp", n)   # or addSourceParticle(xyz)
    A.addTargetParticlesINP("mesh.inp", n)
    A.prcmpt(L, Ncrit, kappa)                 # lvMAX=-1: leaf size criterion
    gemv(A, In, Out)                          # Out[:] = A @ In (complex128)
    CheckFULL(A)                              # sampled FP64 direct-sum check

Differences, by design: errors raise ``DefmmError`` (the reference prints and
exits); every ``gemv`` is correct (the reference's is only on its first call);
``CheckFULL`` samples targets (the reference sums all N x M pairs).
There is no CPU fallback: without the built library or without a CUDA device
the calls that need them raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdefmm_b200.so")
_lib = None

PRECISION_FP64 = 0
PRECISION_MIXED = 1

_INFO = {
    "n_sources": 0, "n_targets": 1, "nlvl": 2, "cpt": 3, "max_stage": 4, "cells_T": 5,
    "cells_S": 6, "slots_S": 7, "slots_T": 8, "far_hf": 9, "far_lf": 10, "near": 11,
    "i_near": 12, "tables": 13, "device_bytes": 14, "list_records": 15, "launches": 16,
    "m2l_targets": 17, "leaf_slots_S": 18, "permuted_spectra": 19, "plan_walk_device": 20, "plan_ms": 21,
    "plan_walk_ms": 22, "m2l_threads": 23, "p2p_blocks_per_sm": 24, "m2l_pairing": 25,
    "layout": 26, "rhs_block": 27, "groups": 28, "m2m_entries": 29, "l2l_entries": 30,
    "p2m_point_slots": 31, "l2p_point_slots": 32, "m2f_slots": 33, "tensor_cores": 34,
    "tree_device": 35, "tree_ms": 36, "rhs_per_cta": 37, "m2l_staging": 38, "m2l_group_list": 39,
}
PHASES = ["p2m", "m2m", "m2f", "m2l", "f2l", "l2l", "l2p", "p2p", "scatter", "total"]


class DefmmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"defmm_b200 error {code}: {msg}")
        self.code = code


def lib():
    """Load the in-tree CUDA library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise DefmmError(-4, f"{_LIB_PATH} is missing: run defmm_b200.build.build()")
        L = ctypes.CDLL(_LIB_PATH)
        vp, dp, ip, i64 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32), ctypes.c_int64
        sig = {
            "defmm_device_count": (ctypes.c_int, []),
            "defmm_create": (vp, []),
            "defmm_destroy": (None, [vp]),
            "defmm_last_error": (ctypes.c_char_p, [vp]),
            "defmm_add_source_particle": (ctypes.c_int, [vp, dp]),
            "defmm_add_target_particle": (ctypes.c_int, [vp, dp]),
            "defmm_add_sources": (ctypes.c_int, [vp, dp, i64]),
            "defmm_add_targets": (ctypes.c_int, [vp, dp, i64]),
            "defmm_load_inp": (ctypes.c_int, [vp, ctypes.c_char_p, i64, ctypes.c_int]),
            "defmm_prcmpt": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
            "defmm_upload": (ctypes.c_int, [vp]),
            "defmm_set_precision": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_gemv": (ctypes.c_int, [vp, dp, dp]),
            "defmm_gemv_device": (ctypes.c_int, [vp, vp, vp, i64, vp]),
            "defmm_gemv_batched": (ctypes.c_int, [vp, i64, dp, dp]),
            "defmm_check_full": (ctypes.c_int, [vp, i64, ctypes.c_uint64, dp]),
            "defmm_direct_noalloc": (ctypes.c_int, [vp, vp, i64, vp, vp]),
            "defmm_info": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(i64)]),
            "defmm_phase_times": (ctypes.c_int, [vp, dp]),
            "defmm_set_profiling": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_set_graphs": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_keep_lists": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_set_plan_device": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_autotune": (ctypes.c_int, [vp, ctypes.c_int, ip]),
            "defmm_set_launch": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
            "defmm_set_m2l_pairing": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_set_blocking": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
            "defmm_dump_m2l": (ctypes.c_int, [vp, vp, vp, vp, ctypes.POINTER(i64)]),
            "defmm_near_digest": (ctypes.c_int, [vp, vp]),
            "defmm_probe_l2_read": (ctypes.c_int, [i64, ctypes.c_int, dp]),
            "defmm_set_rhs_per_cta": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_set_tensor_cores": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_set_m2l_staging": (ctypes.c_int, [vp, ctypes.c_int]),
            "defmm_m2l_schedule": (ctypes.c_int, [vp, ip, ip, ctypes.c_int]),
            "defmm_setup_times": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.POINTER(i64)]),
            "defmm_batch_create": (vp, [i64, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_int]),
            "defmm_batch_launch": (ctypes.c_int, [vp, vp]),
            "defmm_batch_destroy": (None, [vp]),
            "defmm_dump_tree": (ctypes.c_int, [vp, ctypes.c_int, ip, dp, ip, ctypes.POINTER(i64), ip]),
            "defmm_dump_lists": (ctypes.c_int, [vp, ip, ip, ip, ctypes.POINTER(i64)]),
            "defmm_mlp_forward": (ctypes.c_int, [vp, vp, i64, vp, vp, vp, vp]),
            "defmm_mlp_backward": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp, ctypes.c_float, i64, vp, vp, vp,
                                                  vp]),
            "defmm_mlp_adam": (ctypes.c_int, [vp, vp, vp, vp, i64, ctypes.c_float, ctypes.c_float, vp]),
            "defmm_mlp_to_bf16": (ctypes.c_int, [vp, vp, vp]),
            "defmm_mlp_infer_bf16": (ctypes.c_int, [vp, vp, i64, vp, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def probe_l2_read(nbytes=64 << 20, reps=200) -> float:
    """L2-to-SM read bandwidth of the current device, GB/s (defmm_probe_l2_read)."""
    g = ctypes.c_double(0.0)
    st = lib().defmm_probe_l2_read(int(nbytes), int(reps), ctypes.byref(g))
    if st:
        raise DefmmError(st, "L2 bandwidth probe failed")
    return float(g.value)


def device_count() -> int:
    return int(lib().defmm_device_count())


class IBFMM_Mat:
    """FMM operator for exp(i kappa r)/(4 pi r) between source and target
    point clouds (include/interface.hpp:46)."""

    def __init__(self):
        self._h = lib().defmm_create()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.defmm_destroy(h)
            self._h = None

    # -- errors
    def _check(self, st):
        if st != 0:
            raise DefmmError(st, lib().defmm_last_error(self._h).decode())

    # -- particles (interface.hpp:59-98)
    def addSourceParticle(self, part):
        a = np.ascontiguousarray(part, dtype=np.float64).reshape(3)
        self._check(lib().defmm_add_source_particle(self._h, _dp(a)))

    def addTargetParticle(self, part):
        a = np.ascontiguousarray(part, dtype=np.float64).reshape(3)
        self._check(lib().defmm_add_target_particle(self._h, _dp(a)))

    def addSourceParticles(self, pts):
        a = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        self._check(lib().defmm_add_sources(self._h, _dp(a), a.shape[0]))

    def addTargetParticles(self, pts):
        a = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        self._check(lib().defmm_add_targets(self._h, _dp(a), a.shape[0]))

    def addSourceParticlesINP(self, name, nparts):
        self._check(lib().defmm_load_inp(self._h, os.fsencode(name), int(nparts), 0))

    def addTargetParticlesINP(self, name, nparts):
        self._check(lib().defmm_load_inp(self._h, os.fsencode(name), int(nparts), 1))

    # -- precomputation (interface.hpp:100-151)
    def prcmpt(self, L, Ncrit, kappa, lvMAX=-1):
        self._check(lib().defmm_prcmpt(self._h, int(L), int(Ncrit), float(kappa), int(lvMAX)))

    def upload(self):
        self._check(lib().defmm_upload(self._h))

    def set_precision(self, mode):
        if isinstance(mode, str):
            mode = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}[mode]
        self._check(lib().defmm_set_precision(self._h, int(mode)))

    def set_plan_device(self, on=True):
        """Run prcmpt's level walk on the GPU (default) or on the host."""
        self._check(lib().defmm_set_plan_device(self._h, int(bool(on))))

    def autotune(self, reps=2):
        """Pick the fastest launch choices for this operator at its current
        precision (defmm_autotune); returns {"m2l_threads", "m2l_pairing",
        "p2p_blocks_per_sm"}."""
        c = np.zeros(2, dtype=np.int32)
        self._check(lib().defmm_autotune(self._h, int(reps), _ip(c)))
        return {"m2l_threads": int(c[0]), "m2l_pairing": self.info("m2l_pairing"), "p2p_blocks_per_sm": int(c[1])}

    def set_launch(self, m2l_threads=0, p2p_blocks_per_sm=0):
        """Launch choices by hand for the current precision (0: defaults)."""
        self._check(lib().defmm_set_launch(self._h, int(m2l_threads), int(p2p_blocks_per_sm)))

    def set_m2l_pairing(self, on=True):
        """Two target slots per M2L CTA (current precision); results unchanged."""
        self._check(lib().defmm_set_m2l_pairing(self._h, int(bool(on))))

    def set_blocking(self, rhs_block=16, groups=0):
        """Right-hand sides per pass of multi-RHS calls (1..32) and the number
        of direction groups of the grouped layout (0: as memory needs; >= 1:
        about that many, also for single right-hand sides)."""
        self._check(lib().defmm_set_blocking(self._h, int(rhs_block), int(groups)))

    def set_tensor_cores(self, on=True):
        """Mixed precision: P2M on the tensor cores (tcgen05, split TF32)."""
        self._check(lib().defmm_set_tensor_cores(self._h, int(bool(on))))

    def m2l_schedule(self) -> list:
        """(threads, pairing) of the M2L launches per level, current precision."""
        n = int(self.info("nlvl"))
        t, p = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self._check(lib().defmm_m2l_schedule(self._h, _ip(t), _ip(p), n))
        return [(int(a), int(b)) for a, b in zip(t, p)]

    def setup_times(self) -> dict:
        """Seconds per step of the last prcmpt (defmm_setup_times)."""
        n = ctypes.c_int64(0)
        self._check(lib().defmm_setup_times(self._h, None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(int(n.value))
        self._check(lib().defmm_setup_times(self._h, buf, ctypes.byref(n)))
        out = {}
        for line in buf.value.decode().splitlines():
            t, name = line.split("\t", 1)
            out[name] = out.get(name, 0.0) + float(t)
        return out

    def set_m2l_staging(self, on=True):
        """Grouped layout, mixed precision, orders 3-6: M2L staged through
        shared memory by bulk copies with four target slots per CTA, or one
        target slot per CTA (default, faster); bit-identical results."""
        self._check(lib().defmm_set_m2l_staging(self._h, int(bool(on))))

    def set_rhs_per_cta(self, rb=4):
        """Right-hand sides per M2L CTA of the grouped layout (1, 2, 4, 8)."""
        self._check(lib().defmm_set_rhs_per_cta(self._h, int(rb)))

    def set_profiling(self, on=True):
        self._check(lib().defmm_set_profiling(self._h, int(bool(on))))

    def set_graphs(self, on=True):
        self._check(lib().defmm_set_graphs(self._h, int(bool(on))))

    def keep_lists(self, on=True):
        self._check(lib().defmm_keep_lists(self._h, int(bool(on))))

    # -- apply
    def matvec(self, q):
        q = np.ascontiguousarray(q, dtype=np.complex128)
        nrhs = 1 if q.ndim == 1 else q.shape[0]
        out = np.empty((nrhs, self.info("n_targets")), dtype=np.complex128)
        self._check(lib().defmm_gemv_batched(self._h, nrhs, _dp(q.view(np.float64)), _dp(out.view(np.float64))))
        return out[0] if q.ndim == 1 else out

    def matvec_device(self, d_in, d_out, nrhs=1, stream=0):
        """Device pointers (ints, e.g. torch.Tensor.data_ptr()) of complex128
        vectors in user order; enqueued on `stream` without synchronising."""
        self._check(lib().defmm_gemv_device(self._h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                                            int(nrhs), ctypes.c_void_p(stream) if stream else None))

    def check_full(self, nsamples=2000, seed=7):
        err = np.zeros(3)
        self._check(lib().defmm_check_full(self._h, int(nsamples), int(seed), _dp(err)))
        return {"linf": err[0], "l1": err[1], "l2": err[2]}

    def direct_noalloc(self, d_targets, nt, d_out, stream=0):
        """FP64 direct sums at `nt` device target points (nt x 3 float64)
        into `d_out` (nt complex128), charges of the last host matvec; no
        device allocation, nt <= 262144, calls on one device must not
        overlap.  Enqueued on `stream` without synchronising."""
        self._check(lib().defmm_direct_noalloc(self._h, ctypes.c_void_p(d_targets), int(nt),
                                               ctypes.c_void_p(d_out), ctypes.c_void_p(stream) if stream else None))

    # -- introspection
    def info(self, what=None):
        if what is None:
            return {k: self.info(k) for k in _INFO}
        v = ctypes.c_int64(0)
        self._check(lib().defmm_info(self._h, _INFO[what], ctypes.byref(v)))
        return int(v.value)

    def phase_times(self):
        ms = np.zeros(10)
        self._check(lib().defmm_phase_times(self._h, _dp(ms)))
        return dict(zip(PHASES, ms.tolist()))

    def tree(self, which):
        """(cells_int (n,8), cells_dbl (n,4), dirs, perm) in the reference's
        cell-array layout (SourceRoot/TargetRoot, interface.hpp:174-175)."""
        w = 0 if which == "T" else 1
        n = self.info("cells_T" if w == 0 else "cells_S")
        ci = np.zeros((n, 8), np.int32)
        cd = np.zeros((n, 4), np.float64)
        nd = ctypes.c_int64(0)
        self._check(lib().defmm_dump_tree(self._h, w, None, None, None, ctypes.byref(nd), None))
        dirs = np.zeros(nd.value, np.int32)
        npart = self.info("n_targets" if w == 0 else "n_sources")
        perm = np.zeros(npart, np.int32)
        self._check(lib().defmm_dump_tree(self._h, w, _ip(ci), _dp(cd), _ip(dirs), ctypes.byref(nd), _ip(perm)))
        return ci, cd, dirs, perm

    def lists(self):
        n = (ctypes.c_int64 * 3)()
        self._check(lib().defmm_dump_lists(self._h, None, None, None, n))
        fh = np.zeros((n[0], 6), np.int32)
        fl = np.zeros((n[1], 5), np.int32)
        nr = np.zeros((n[2], 2), np.int32)
        self._check(lib().defmm_dump_lists(self._h, _ip(fh), _ip(fl), _ip(nr), n))
        return nr, fh, fl

    def m2l_entries(self):
        """(ptr, src, tab): the M2L work per target slot as the matvec runs
        it (defmm_dump_m2l)."""
        n = (ctypes.c_int64 * 2)()
        self._check(lib().defmm_dump_m2l(self._h, None, None, None, n))
        ptr = np.zeros(n[0], np.int64)
        src = np.zeros(n[1], np.int32)
        tab = np.zeros(n[1], np.uint32)
        self._check(lib().defmm_dump_m2l(self._h, ptr.ctypes.data, src.ctypes.data, tab.ctypes.data, n))
        return ptr, src, tab

    def near_digest(self):
        """26 fingerprints of the near-field work lists as the matvec runs
        them (defmm_near_digest)."""
        d = np.zeros(26, np.uint64)
        self._check(lib().defmm_near_digest(self._h, d.ctypes.data))
        return d


class MultiFreqMat:
    """The reference's multi-frequency kernel (thetis_kernels.hpp:36)
        G(R) = sum_{a in (1, 3.6, 2, 8)} exp(i (kappa / a) R) / (4 pi R),
    applied as the sum of four Helmholtz operators, one per wavenumber, each
    with the tree, cones and lists of its own wavenumber (the reference
    defines the kernel but builds its transfer spectra and cones for one
    Helmholtz wavenumber only, interface.hpp:127, M2L.hpp:181).  Same calls
    as IBFMM_Mat for building and applying."""

    DIVISORS = (1.0, 3.6, 2.0, 8.0)

    def __init__(self):
        self.parts = [IBFMM_Mat() for _ in self.DIVISORS]

    def addSourceParticles(self, pts):
        for A in self.parts:
            A.addSourceParticles(pts)

    def addTargetParticles(self, pts):
        for A in self.parts:
            A.addTargetParticles(pts)

    def set_precision(self, mode):
        for A in self.parts:
            A.set_precision(mode)

    def prcmpt(self, L, Ncrit, kappa, lvMAX=-1):
        for A, a in zip(self.parts, self.DIVISORS):
            A.prcmpt(L, Ncrit, kappa / a, lvMAX)

    def matvec(self, q):
        out = self.parts[0].matvec(q)
        for A in self.parts[1:]:
            out = out + A.matvec(q)
        return out


class Batch:
    """Several operators applied by one graph launch (defmm_batch_*): ops[i]
    maps the device vector at d_in[i] to d_out[i] (pointers as ints, e.g.
    torch.Tensor.data_ptr()).  Creating the batch runs every member once.
    `lanes` chains run concurrently; the matvecs of one chain run in turn."""

    def __init__(self, ops, d_in, d_out, lanes=1):
        n = len(ops)
        if not (n == len(d_in) == len(d_out)) or n == 0:
            raise ValueError("one input and one output per operator")
        hs = (ctypes.c_void_p * n)(*[op._h for op in ops])
        ins = (ctypes.c_void_p * n)(*d_in)
        outs = (ctypes.c_void_p * n)(*d_out)
        self._ops = list(ops)  # members must outlive the batch
        if lanes < 1:
            raise ValueError("lanes must be >= 1")
        self._b = lib().defmm_batch_create(n, hs, ins, outs, int(lanes))
        if not self._b:
            msgs = "; ".join(lib().defmm_last_error(op._h).decode() for op in ops if lib().defmm_last_error(op._h))
            raise DefmmError(-4, "batch creation failed" + (": " + msgs if msgs else ""))

    def launch(self, stream=0):
        st = lib().defmm_batch_launch(self._b, ctypes.c_void_p(stream) if stream else None)
        if st != 0:
            raise DefmmError(st, "batch launch failed")

    def __del__(self):
        if getattr(self, "_b", None):
            lib().defmm_batch_destroy(self._b)
            self._b = None


def SourceRoot(A):
    return A.tree("S")


def TargetRoot(A):
    return A.tree("T")


def gemv(A, In, Out):
    """friend gemv(IBFMM_Mat&, Vecc& In, Vecc& Out) (interface.hpp:153-170)."""
    Out[...] = A.matvec(In)


def CheckFULL(A, nsamples=2000, seed=7):
    """friend CheckFULL(IBFMM_Mat&) (interface.hpp:178-221), sampled targets."""
    e = A.check_full(nsamples, seed)
    print(f"Relative L^oo norm: {e['linf']}")
    print(f"Relative L^1  norm: {e['l1']}")
    print(f"Relative L^2  norm: {e['l2']}")
    return e
