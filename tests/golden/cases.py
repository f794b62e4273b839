"""Seeded parity cases shared by the fixture generator and the tests.

Each case exercises a different part of the reference's method:

* ``cube20k``   -- the cube-surface workload (N = 20,000, k = 2 pi 16/sqrt 3,
  order 4, leaf size 64): all levels high-frequency (directional).
* ``cube_lf``   -- the same surface at 2 wavelengths, order 5, leaf size 32:
  low-frequency levels under the directional ones (lfM2M, lf2hfM2M,
  hf2lfL2L, LF M2L with its own tables).
* ``fixed_depth`` -- fixed-depth tree (prcmpt's lvMAX = 5) at 4 wavelengths.
* ``blobs_sphere`` -- distinct sources (Gaussian blobs) and targets (a
  sphere), order 4, leaf size 40.
* ``sphere_l6`` -- sphere surface, 30,000 points, 16 wavelengths, order 6.
* ``cube_laplace`` -- cube surface at k = 0: the reference's Laplace kernel
  1/(4 pi r) (thetis_kernels.hpp:35) through the same method, every level
  low-frequency.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

from defmm_b200 import workloads as W  # noqa: E402

CASES = ["cube20k", "cube_lf", "fixed_depth", "blobs_sphere", "sphere_l6", "cube_laplace"]


def case_inputs(name):
    """(src, trg, q, L, ncrit, kappa, lvmax) for a named case."""
    if name == "cube20k":
        w = W.cube_surface()
        return w.points, w.points, W.charges(w.n, 5), w.order, w.ncrit, w.kappa, -1
    if name == "cube_lf":
        p = W.cube_surface(20000, seed=3).points
        return p, p, W.charges(len(p), 5), 5, 32, 2 * math.pi * 2 / math.sqrt(3), -1
    if name == "fixed_depth":
        p = W.cube_surface(20000, seed=3).points
        return p, p, W.charges(len(p), 5), 4, 32, 2 * math.pi * 4 / math.sqrt(3), 5
    if name == "blobs_sphere":
        src = W.gaussian_blobs(15000, seed=2, wavelengths=6).points
        trg = W.sphere_surface(8000, seed=4).points * 0.45
        return src, trg, W.charges(len(src), 5), 4, 40, 2 * math.pi * 6 / math.sqrt(3), -1
    if name == "sphere_l6":
        p = W.sphere_surface(30000, seed=9).points
        return p, p, W.charges(len(p), 5), 6, 64, 2 * math.pi * 8, -1
    if name == "cube_laplace":
        p = W.cube_surface(20000, seed=2).points
        return p, p, W.charges(len(p), 5), 4, 64, 0.0, -1
    raise KeyError(name)
