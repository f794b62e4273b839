"""Test infrastructure (oracle only): ctypes wrapper of the C++ restatement of
the reference defmm FMM (oracle/defmm_oracle.cpp -> oracle/_ref/libdefmm_oracle.so).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libdefmm_oracle.so")

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "restated"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [dp, ctypes.c_int64, dp, ctypes.c_int64, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.oracle_status.argtypes = [ctypes.c_void_p]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_gemv.argtypes = [ctypes.c_void_p, dp, dp]
        L.oracle_info.restype = ctypes.c_int64
        L.oracle_info.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_cells.argtypes = [ctypes.c_void_p, ctypes.c_int, ip, dp]
        L.oracle_dirs.restype = ctypes.c_int64
        L.oracle_dirs.argtypes = [ctypes.c_void_p, ctypes.c_int, ip]
        L.oracle_perm.argtypes = [ctypes.c_void_p, ctypes.c_int, ip]
        L.oracle_lists.argtypes = [ctypes.c_void_p, ip, ip, ip]
        L.oracle_table.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, dp]
        L.oracle_direction.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.oracle_direct.argtypes = [dp, ctypes.c_int64, dp, dp, ctypes.c_int64,
                                    ctypes.c_double, dp]
        L.oracle_create_opt.restype = ctypes.c_void_p
        L.oracle_create_opt.argtypes = [dp, ctypes.c_int64, dp, ctypes.c_int64, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.oracle_digest_records.argtypes = [ip, ctypes.c_int64, ctypes.c_int, u64p]
        L.oracle_lists_digest.argtypes = [ctypes.c_void_p, ctypes.c_int, u64p]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


class OracleFMM:
    """CPU restatement of IBFMM_Mat<3>: build (prcmpt) at construction."""

    def __init__(self, src, trg, L, ncrit, kappa, lvmax=-1, lists_only=False):
        """lists_only: build the trees, cones, effective directions and
        interaction lists only (no matvec possible)."""
        self.src = np.ascontiguousarray(src, dtype=np.float64)
        self.trg = np.ascontiguousarray(trg, dtype=np.float64)
        self.L, self.ncrit, self.kappa = L, ncrit, kappa
        self._h = lib().oracle_create_opt(_dp(self.src), self.src.shape[0], _dp(self.trg),
                                          self.trg.shape[0], L, ncrit, kappa, lvmax, int(bool(lists_only)))
        self.status = lib().oracle_status(self._h)

    def lists_digest(self):
        """Order-independent digests {near, far_hf, far_lf} of the lists
        (see records_digest)."""
        out = {}
        for w, name in enumerate(["near", "far_hf", "far_lf"]):
            d = np.zeros(3, np.uint64)
            lib().oracle_lists_digest(self._h, w, d.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
            out[name] = [int(x) for x in d]
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def info(self):
        names = ["nlvl", "cpt", "max_stage", "n_far_hf", "n_far_lf", "n_near",
                 "cells_T", "cells_S", "nsrc_exp", "ntrg_exp", "hf_tables"]
        return {n: int(lib().oracle_info(self._h, i)) for i, n in enumerate(names)}

    def gemv(self, q):
        q = np.ascontiguousarray(q, dtype=np.complex128)
        p = np.zeros(self.trg.shape[0], dtype=np.complex128)
        st = lib().oracle_gemv(self._h, _dp(q.view(np.float64)), _dp(p.view(np.float64)))
        if st:
            raise RuntimeError(f"oracle gemv status {st}")
        return p

    def tree(self, which):  # which: "T" or "S"
        w = 0 if which == "T" else 1
        n = self.info()["cells_T" if w == 0 else "cells_S"]
        ci = np.zeros((n, 8), np.int32)
        cd = np.zeros((n, 4), np.float64)
        lib().oracle_cells(self._h, w, _ip(ci), _dp(cd))
        nd = lib().oracle_dirs(self._h, w, None)
        dirs = np.zeros(nd, np.int32)
        lib().oracle_dirs(self._h, w, _ip(dirs))
        npart = (self.trg if w == 0 else self.src).shape[0]
        perm = np.zeros(npart, np.int32)
        lib().oracle_perm(self._h, w, _ip(perm))
        return ci, cd, dirs, perm

    def lists(self):
        inf = self.info()
        near = np.zeros((inf["n_near"], 2), np.int32)
        fh = np.zeros((inf["n_far_hf"], 6), np.int32)
        fl = np.zeros((inf["n_far_lf"], 5), np.int32)
        lib().oracle_lists(self._h, _ip(near), _ip(fh), _ip(fl))
        return near, fh, fl

    def table(self, lvl, iz):
        out = np.zeros((2 * self.L - 1) ** 3, np.complex128)
        ok = lib().oracle_table(self._h, lvl, iz, _dp(out.view(np.float64)))
        return out if ok else None

    def direction(self, stage, d):
        out = np.zeros(3)
        lib().oracle_direction(self._h, stage, d, _dp(out))
        return out


def records_digest(rec):
    """[count, sum h1, sum h2] (mod 2^64) of the rows of an int32 record
    array: equal for equal multisets of rows, whatever their order."""
    rec = np.ascontiguousarray(rec, dtype=np.int32)
    d = np.zeros(3, np.uint64)
    n = rec.shape[0]
    w = rec.shape[1] if rec.ndim == 2 else 1
    lib().oracle_digest_records(_ip(rec.reshape(-1)) if n else None, n, w,
                                d.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return [int(x) for x in d]


def direct(src, q, trg, kappa):
    """FP64 direct sum p(x) = sum_j q_j exp(i k r)/(4 pi r), r > 1e-8 only."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    trg = np.ascontiguousarray(trg, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.complex128)
    out = np.zeros(trg.shape[0], np.complex128)
    lib().oracle_direct(_dp(src), src.shape[0], _dp(q.view(np.float64)), _dp(trg),
                        trg.shape[0], kappa, _dp(out.view(np.float64)))
    return out
