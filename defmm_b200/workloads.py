"""Seeded synthetic point sets and charge vectors for the matvec workloads.

No public dataset is involved: every workload is generated here from a seed
with numpy's PCG64 (``numpy.random.default_rng(seed)``).  The shapes follow
the workloads the matvec is measured on:

* ``cube_surface``  -- N points on the surface of [-0.5, 0.5]^3, 70 % uniform
  over the six faces and 30 % within 0.05 of the twelve edges (a non-uniform
  surface like the reference's refined-cube mesh, mesh/refinedcube.inp);
  wavenumber such that the cube diagonal spans 16 wavelengths
  (k = 2*pi*16/sqrt(3)); order 4, leaf size 64.
* ``sphere_surface`` -- N points uniform on the unit sphere (normalised
  Gaussian samples); k such that the diameter (2) spans 128 wavelengths
  (k = 2*pi*64); order 5, leaf size 64.
* ``spheroid``      -- prolate spheroid with semi-axes (1, 0.5, 0.25) and
  density proportional to 1 + 4|z| (rejection sampling); k such that the long
  axis (2) spans 256 wavelengths.
* ``gaussian_blobs`` -- isotropic Gaussian blobs inside the unit cube.
* ``mixture``       -- 40 % cube surface, 30 % sphere surface of radius 0.4,
  30 % Gaussian blobs with sigma in [0.01, 0.1]; k such that the cube
  diagonal (sqrt 3) spans 512 wavelengths; order 6, leaf size 96.

Charges are complex with real and imaginary parts uniform in [-1, 1].
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Workload:
    name: str
    points: np.ndarray  # (N, 3) float64
    kappa: float
    order: int
    ncrit: int

    @property
    def n(self) -> int:
        return int(self.points.shape[0])


def _face_points(rng, n):
    """Uniform points on the surface of [-0.5, 0.5]^3 (six equal faces)."""
    face = rng.integers(0, 6, size=n)
    uv = rng.uniform(-0.5, 0.5, size=(n, 2))
    axis = face // 2
    sign = np.where(face % 2 == 0, -0.5, 0.5)
    p = np.empty((n, 3))
    for a in range(3):
        sel = axis == a
        others = [b for b in range(3) if b != a]
        p[sel, a] = sign[sel]
        p[sel, others[0]] = uv[sel, 0]
        p[sel, others[1]] = uv[sel, 1]
    return p


def _edge_points(rng, n, width=0.05):
    """Points on the cube surface within `width` of one of its 12 edges."""
    edge = rng.integers(0, 12, size=n)
    along = rng.uniform(-0.5, 0.5, size=n)
    off = rng.uniform(0.0, width, size=n)
    which = rng.integers(0, 2, size=n)  # which of the two adjacent faces
    p = np.empty((n, 3))
    for e in range(12):
        sel = edge == e
        a = e // 4  # axis the edge runs along
        s1 = -0.5 if (e & 1) == 0 else 0.5
        s2 = -0.5 if (e & 2) == 0 else 0.5
        b, c = [x for x in range(3) if x != a]
        p[sel, a] = along[sel]
        # on face b = s1: move from the edge along c towards the face centre
        w = which[sel] == 0
        pb = np.where(w, s1, s1 - np.sign(s1) * off[sel])
        pc = np.where(w, s2 - np.sign(s2) * off[sel], s2)
        p[sel, b] = pb
        p[sel, c] = pc
    return p


def cube_surface(n: int = 20_000, seed: int = 0) -> Workload:
    rng = np.random.default_rng(seed)
    n_edge = int(round(0.3 * n))
    pts = np.concatenate([_face_points(rng, n - n_edge), _edge_points(rng, n_edge)])
    pts = pts[rng.permutation(n)]
    return Workload("cube_surface", np.ascontiguousarray(pts),
                    2.0 * math.pi * 16.0 / math.sqrt(3.0), 4, 64)


def sphere_surface(n: int = 2_000_000, seed: int = 0, wavelengths: float = 128.0,
                   order: int = 5, ncrit: int = 64) -> Workload:
    rng = np.random.default_rng(seed)
    g = rng.standard_normal(size=(n, 3))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    return Workload("sphere_surface", np.ascontiguousarray(g),
                    2.0 * math.pi * wavelengths / 2.0, order, ncrit)


def spheroid(n: int = 4_000_000, seed: int = 0, order: int = 6, ncrit: int = 96,
             wavelengths: float = 256.0) -> Workload:
    rng = np.random.default_rng(seed)
    a = np.array([1.0, 0.5, 0.25])
    out = []
    need = n
    while need > 0:
        g = rng.standard_normal(size=(2 * need + 1024, 3))
        g /= np.linalg.norm(g, axis=1, keepdims=True)
        p = g * a
        # density proportional to 1 + 4|z| on the surface; accept with ratio
        keep = rng.uniform(0.0, 1.0 + 4.0 * a[2], size=p.shape[0]) < 1.0 + 4.0 * np.abs(p[:, 2])
        out.append(p[keep][:need])
        need -= out[-1].shape[0]
    pts = np.concatenate(out)[:n]
    return Workload("spheroid", np.ascontiguousarray(pts),
                    2.0 * math.pi * wavelengths / 2.0, order, ncrit)


def gaussian_blobs(n: int, seed: int = 0, nblobs: int = 8, sigma: float = 0.05,
                   wavelengths: float = 32.0, order: int = 4, ncrit: int = 64) -> Workload:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, size=(nblobs, 3)) - 0.5
    which = rng.integers(0, nblobs, size=n)
    pts = centres[which] + sigma * rng.standard_normal(size=(n, 3))
    pts = np.clip(pts, -0.5, 0.5)
    return Workload("gaussian_blobs", np.ascontiguousarray(pts),
                    2.0 * math.pi * wavelengths / math.sqrt(3.0), order, ncrit)


def mixture(n: int = 8_000_000, seed: int = 0, wavelengths: float = 512.0, order: int = 6,
            ncrit: int = 96, nblobs: int = 16) -> Workload:
    """40 % of the points uniform on the surface of [-0.5, 0.5]^3, 30 % uniform
    on the sphere of radius 0.4 about the origin, 30 % in `nblobs` isotropic
    Gaussian blobs (centres uniform in [-0.3, 0.3]^3, sigma log-uniform in
    [0.01, 0.1], clipped to the cube); the diagonal sqrt(3) spans
    `wavelengths` wavelengths."""
    rng = np.random.default_rng(seed)
    n_cube = int(round(0.4 * n))
    n_sph = int(round(0.3 * n))
    n_blob = n - n_cube - n_sph
    cube = _face_points(rng, n_cube)
    g = rng.standard_normal(size=(n_sph, 3))
    sph = 0.4 * g / np.linalg.norm(g, axis=1, keepdims=True)
    centres = rng.uniform(-0.3, 0.3, size=(nblobs, 3))
    sig = np.exp(rng.uniform(math.log(0.01), math.log(0.1), size=nblobs))
    which = rng.integers(0, nblobs, size=n_blob)
    blob = np.clip(centres[which] + sig[which, None] * rng.standard_normal(size=(n_blob, 3)), -0.5, 0.5)
    pts = np.concatenate([cube, sph, blob])[rng.permutation(n)]
    return Workload("mixture", np.ascontiguousarray(pts), 2.0 * math.pi * wavelengths / math.sqrt(3.0), order, ncrit)


def ragged_problems(count: int = 48, seed: int = 0) -> list:
    """Independent problems of uneven size for one batched launch: N
    log-uniform in [5,000, 250,000]; geometry cycling cube surface / sphere
    surface / 8 Gaussian blobs (sigma 0.05) in the unit cube; 8-128
    wavelengths across the diameter (log-uniform, capped so that the surface
    keeps >= 25 points per square wavelength and the tree reaches a level
    with far-field work); order 4-6; leaf size 64."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(5e3), math.log(2.5e5)))))
        wl = math.exp(rng.uniform(math.log(8.0), math.log(128.0)))
        wl = max(2.0, min(wl, math.sqrt(n / (25.0 * math.pi))))
        order = 4 + i % 3
        g = i % 3
        if g == 0:
            c = cube_surface(n, seed=seed * 1000 + i)
            w = Workload("cube_surface", c.points, 2.0 * math.pi * wl / math.sqrt(3.0), order, 64)
        elif g == 1:
            w = sphere_surface(n, seed=seed * 1000 + i, wavelengths=wl, order=order)
        else:
            w = gaussian_blobs(n, seed=seed * 1000 + i, wavelengths=wl, order=order)
        out.append(w)
    return out


def charges(n: int, seed: int = 1, nrhs: int | None = None) -> np.ndarray:
    """Complex charges, real and imaginary parts uniform in [-1, 1]."""
    rng = np.random.default_rng(seed)
    shape = (n,) if nrhs is None else (nrhs, n)
    return (rng.uniform(-1.0, 1.0, size=shape)
            + 1j * rng.uniform(-1.0, 1.0, size=shape)).astype(np.complex128)


def sample_targets(n: int, m: int = 2000, seed: int = 7) -> np.ndarray:
    """Seeded random target indices for direct-sum accuracy checks."""
    rng = np.random.default_rng(seed)
    m = min(m, n)
    return np.sort(rng.choice(n, size=m, replace=False)).astype(np.int64)
