"""Synthetic triangulations in BEST's input format, for the benchmark and the parity tests.

BEST reads a header ``NAR [TRUEAREA TRUEVOL]`` and then one line of 9 reals per triangle
(best/best.f:189-221); vertices are stored per triangle, and COMPON (best/compon.f90:19-116) finds
closed surfaces by matching vertex coordinates exactly, so every generator here builds an indexed
mesh first and writes each shared vertex with bit-identical coordinates.  Triangles are ordered
counter-clockwise seen from outside, as in the reference's example meshes, so BEST's normal
(v3 - v1) x (v2 - v1) points inward.

Workloads (radii in Angstrom):
  icosphere(3, 20)          subdivided icosahedron, N = 1,280, on a sphere of radius 20
  ellipsoid(16, seed=0)     geodesic frequency 16 (N = 5,120) on the 30/20/12 ellipsoid, vertices
                            moved along the normal by U(-2%, +2%) of the local radius
  star(32, seed=1)          r = 25 (1 + sum_{l=2..8} sum_m a_lm Y_lm), a_lm ~ N(0, (0.08/l)^2),
                            geodesic frequency 32 (N = 20,480) or 45 (N = 40,500)
  ellipsoid series f in {11,12,14,16,18,20,22,23}: N = 2,420 .. 10,580
"""
from __future__ import annotations

import math

import numpy as np


def _icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v, f


def _orient_outward(verts, faces):
    """Counter-clockwise seen from outside: (v2-v1) x (v3-v1) points away from the origin."""
    a, b, c = verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]
    nrm = np.cross(b - a, c - a)
    flip = np.einsum("ij,ij->i", nrm, (a + b + c) / 3.0) < 0
    faces = faces.copy()
    faces[flip, 1], faces[flip, 2] = faces[flip, 2].copy(), faces[flip, 1].copy()
    return faces


def geodesic_unit(freq):
    """Geodesic sphere of frequency ``freq``: each icosahedron face split into freq^2 triangles on a
    barycentric grid, vertices projected to the unit sphere.  Returns (verts (V,3), faces (20 f^2, 3))
    with V = 10 f^2 + 2 and shared vertices deduplicated."""
    iv, ifc = _icosahedron()
    keys = {}
    verts = []

    def vid(p):
        q = p / np.linalg.norm(p)
        k = tuple(np.round(q * 1e9).astype(np.int64))
        if k not in keys:
            keys[k] = len(verts)
            verts.append(q)
        return keys[k]

    faces = []
    f = freq
    for (ia, ib, ic) in ifc:
        A, B, C = iv[ia], iv[ib], iv[ic]
        idx = {}
        for i in range(f + 1):
            for j in range(f + 1 - i):
                idx[(i, j)] = vid((i * B + j * C + (f - i - j) * A) / f)
        for i in range(f):
            for j in range(f - i):
                faces.append((idx[(i, j)], idx[(i + 1, j)], idx[(i, j + 1)]))
                if i + j < f - 1:
                    faces.append((idx[(i + 1, j)], idx[(i + 1, j + 1)], idx[(i, j + 1)]))
    verts = np.array(verts)
    faces = _orient_outward(verts, np.array(faces, dtype=np.int64))
    return verts, faces


def icosphere_unit(level):
    """Icosahedron subdivided ``level`` times (each triangle into 4), projected to the unit sphere:
    20 * 4^level triangles."""
    v, f = _icosahedron()
    verts = [p for p in v]
    for _ in range(level):
        mid = {}
        nf = []

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                mid[k] = len(verts) - 1
            return mid[k]

        for (a, b, c) in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = np.array(nf, dtype=np.int64)
    verts = np.array(verts)
    return verts, _orient_outward(verts, f)


def to_triangles(verts, faces):
    """Per-triangle rows of 9 coordinates (BEST's V1, V2, V3 by row)."""
    return np.ascontiguousarray(np.concatenate([verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]], axis=1))


def mesh_area_volume(verts, faces):
    a, b, c = verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]
    area = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum()
    vol = np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0
    return float(area), float(abs(vol))


def ellipsoid_area(a, b, c, nt=400, nphi=800):
    """Surface area of the ellipsoid x^2/a^2 + y^2/b^2 + z^2/c^2 = 1 by Gauss-Legendre quadrature in
    (cos theta, phi) of |r_theta x r_phi|."""
    u, wu = np.polynomial.legendre.leggauss(nt)  # u = cos(theta)
    ph = (np.arange(nphi) + 0.5) * (2 * math.pi / nphi)
    U, P = np.meshgrid(u, ph, indexing="ij")
    S = np.sqrt(1 - U * U)
    # r = (a S cos p, b S sin p, c U); dA = |r_u x r_p| du dp
    ru = np.stack([-a * U / S * np.cos(P), -b * U / S * np.sin(P), c * np.ones_like(U)], -1)
    rp = np.stack([-a * S * np.sin(P), b * S * np.cos(P), np.zeros_like(U)], -1)
    dA = np.linalg.norm(np.cross(ru, rp), axis=-1)
    return float((dA * wu[:, None]).sum() * (2 * math.pi / nphi))


def icosphere(level=3, radius=20.0):
    """Configuration C1: (tri (N,9), truearea, truevol) with the exact sphere area and volume."""
    v, f = icosphere_unit(level)
    return to_triangles(v * radius, f), 4 * math.pi * radius ** 2, 4 * math.pi * radius ** 3 / 3


def ellipsoid(freq=16, axes=(30.0, 20.0, 12.0), jitter=0.02, seed=0):
    """Configuration C2/C4: geodesic sphere mapped to the ellipsoid, each vertex moved along the
    ellipsoid normal by U(-jitter, +jitter) of its distance from the centre (numpy default_rng(seed)).
    truearea is the smooth ellipsoid's area (quadrature), truevol 4/3 pi a b c."""
    p, f, ta, tv = ellipsoid_vf(freq, axes, jitter, seed)
    return to_triangles(p, f), ta, tv


def ellipsoid_vf(freq=16, axes=(30.0, 20.0, 12.0), jitter=0.02, seed=0):
    """ellipsoid() as shared vertices and faces: (vertices (nv, 3), faces (N, 3), truearea, truevol)."""
    a, b, c = axes
    v, f = geodesic_unit(freq)
    p = v * np.array(axes)
    nrm = p / np.array([a * a, b * b, c * c])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    rng = np.random.default_rng(seed)
    d = rng.uniform(-jitter, jitter, size=len(p)) * np.linalg.norm(p, axis=1)
    p = p + d[:, None] * nrm
    return p, f, ellipsoid_area(a, b, c), 4 * math.pi * a * b * c / 3


def corner_to_vertex(grad, faces, nverts):
    """Sums per-corner gradients (..., N, 3 corners, 3) onto shared vertices: (..., nverts, 3)."""
    grad = np.asarray(grad)
    out = np.zeros(grad.shape[:-3] + (nverts, 3))
    for corner in range(3):
        np.add.at(out, (Ellipsis, faces[:, corner], slice(None)), grad[..., :, corner, :])
    return out


def _real_ylm(l, m, theta, phi):
    from scipy.special import sph_harm_y
    if m == 0:
        return np.real(sph_harm_y(l, 0, theta, phi))
    if m > 0:
        return math.sqrt(2) * (-1) ** m * np.real(sph_harm_y(l, m, theta, phi))
    return math.sqrt(2) * (-1) ** m * np.imag(sph_harm_y(l, -m, theta, phi))


def star(freq=32, radius=25.0, lmax=8, amp=0.08, seed=1):
    """Configuration C3: star-shaped body r(theta, phi) = R (1 + sum a_lm Y_lm), l = 2..lmax, with
    a_lm ~ N(0, (amp/l)^2) from numpy default_rng(seed), meshed as a geodesic sphere of frequency
    ``freq``.  truearea/truevol are the mesh's own (the run uses no area correction)."""
    v, f = geodesic_unit(freq)
    theta = np.arccos(np.clip(v[:, 2], -1, 1))
    phi = np.arctan2(v[:, 1], v[:, 0])
    rng = np.random.default_rng(seed)
    s = np.zeros(len(v))
    for l in range(2, lmax + 1):
        for m in range(-l, l + 1):
            s += rng.normal(0.0, amp / l) * _real_ylm(l, m, theta, phi)
    p = v * (radius * (1.0 + s))[:, None]
    area, vol = mesh_area_volume(p, f)
    return to_triangles(p, f), area, vol


SERIES_FREQS = (11, 12, 14, 16, 18, 20, 22, 23)


def write_best(path, tri, truearea=None, truevol=None):
    """Writes a BEST input file (header, then 9 coordinates per triangle, full precision)."""
    with open(path, "w") as fh:
        if truearea is None:
            fh.write(f"{len(tri)}\n")
        else:
            fh.write(f"{len(tri)} {truearea!r} {truevol!r}\n")
        for row in tri:
            fh.write(" ".join(repr(float(x)) for x in row) + "\n")
