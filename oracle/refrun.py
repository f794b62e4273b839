"""Test infrastructure (oracle only): run the reference defmm binary built by
oracle/Makefile (``oracle/_ref/defmm_ref``) on one case and load its dumps.

The binary wraps the reference's public API unmodified
(include/interface.hpp:46-170: addSourceParticle / addTargetParticle /
prcmpt / gemv); see oracle/ref_harness.cpp.  Only tests/, bench.py's
reference arm and fixture generation may use this module.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "defmm_ref")
REF_BIN_FAST = os.path.join(HERE, "_ref", "defmm_ref_fast")


def available(fast: bool = False) -> bool:
    return os.path.exists(REF_BIN_FAST if fast else REF_BIN)


def write_case(path, src, trg, q, L, ncrit, kappa, lvmax=-1):
    src = np.ascontiguousarray(src, dtype=np.float64)
    trg = np.ascontiguousarray(trg, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.complex128)
    with open(path, "wb") as f:
        f.write(b"DFMMIN01")
        f.write(struct.pack("<qqiiiid", src.shape[0], trg.shape[0], L, ncrit, lvmax, 0, kappa))
        f.write(src.tobytes())
        f.write(trg.tobytes())
        f.write(q.view(np.float64).tobytes())


@dataclass
class RefTree:
    cells_int: np.ndarray  # (nc, 8): idx0 idx1 idx2 lvl nprt ind nson nexp
    cells_dbl: np.ndarray  # (nc, 4): ctr0 ctr1 ctr2 rad
    sons: np.ndarray
    dirs: np.ndarray
    perm: np.ndarray       # tree-order position -> user index


@dataclass
class RefResult:
    pot: np.ndarray
    S: RefTree
    T: RefTree
    near: np.ndarray | None
    far_hf: np.ndarray | None
    far_lf: np.ndarray | None
    summary: dict = field(default_factory=dict)
    stdout: str = ""


def _load_tree(d, tag):
    ci = np.fromfile(os.path.join(d, f"cells_{tag}_int.bin"), dtype=np.int32).reshape(-1, 8)
    cd = np.fromfile(os.path.join(d, f"cells_{tag}_dbl.bin"), dtype=np.float64).reshape(-1, 4)
    sons = np.fromfile(os.path.join(d, f"sons_{tag}.bin"), dtype=np.int32)
    dirs = np.fromfile(os.path.join(d, f"dirs_{tag}.bin"), dtype=np.int32)
    perm = np.fromfile(os.path.join(d, f"perm_{tag}.bin"), dtype=np.int32)
    return RefTree(ci, cd, sons, dirs, perm)


def run(src, trg, q, L, ncrit, kappa, lvmax=-1, lists=True, fast=False, timeout=3600):
    """Run the reference once (one matvec per process: the reference's gemv
    accumulates into non-leaf expansions that it never resets,
    include/interface.hpp:159, so only its first call is valid)."""
    binary = REF_BIN_FAST if fast else REF_BIN
    if not os.path.exists(binary):
        raise FileNotFoundError(f"{binary} not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory(prefix="defmm_ref_") as d:
        case = os.path.join(d, "case.bin")
        write_case(case, src, trg, q, L, ncrit, kappa, lvmax)
        args = [binary, case, d] + ([] if lists else ["nolists"])
        cp = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
        if cp.returncode != 0:
            raise RuntimeError(f"reference failed ({cp.returncode}): {cp.stdout[-2000:]} {cp.stderr[-2000:]}")
        pot = np.fromfile(os.path.join(d, "pot.bin"), dtype=np.float64).view(np.complex128)
        S = _load_tree(d, "S")
        T = _load_tree(d, "T")
        near = far_hf = far_lf = None
        if lists:
            near = np.fromfile(os.path.join(d, "near.bin"), dtype=np.int32).reshape(-1, 2)
            far_hf = np.fromfile(os.path.join(d, "far_hf.bin"), dtype=np.int32).reshape(-1, 6)
            far_lf = np.fromfile(os.path.join(d, "far_lf.bin"), dtype=np.int32).reshape(-1, 5)
        summary = {}
        with open(os.path.join(d, "summary.txt")) as f:
            for line in f:
                k, v = line.strip().split("=", 1)
                summary[k] = float(v)
        return RefResult(pot, S, T, near, far_hf, far_lf, summary, cp.stdout)
