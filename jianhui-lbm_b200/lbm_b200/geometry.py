"""Seeded synthetic porous geometries and the reference's geometry file formats.

In-memory masks are ``uint8`` arrays of shape ``(nz, ny, nx)`` (x fastest in
memory), 0 = pore, 1 = solid -- the token order of the reference's ASCII
geometry files (Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp:935-943,
Accessories/Boundary_Generation.m:25-31).

File formats (both read by the reference's `Parallelize_Geometry`):

* ASCII (``decbin == 0``): one integer per whitespace-separated token, loop
  order k outer, j, i inner (x fastest).  SP3 reads every token as-is and
  treats any non-zero value as solid (SP3:938-943, 3818-3819); the slab
  solver SP skips tokens other than 0/1 (Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars.cpp:1026-1030).
* binary (``decbin == 1``): raw native-endian int32 in C order ``[i][j][k]``
  (z fastest), read with one ``fin.read`` (SP3:960).

Generators follow the workloads the benchmark configurations describe:
overlapping spheres (cell inside when its centre is within distance <= r of
the sphere centre, periodic wrap; the reference's own convention in
Accessories/Boundary_Generation.m:13), added one by one until the pore
fraction reaches the target, and random straight cylinders.
"""
from __future__ import annotations

import os
import numpy as np

__all__ = [
    "overlapping_spheres",
    "random_cylinders",
    "blob_phase_field",
    "write_ascii",
    "write_binary",
    "read_ascii",
    "read_binary",
    "porosity",
]


def porosity(mask: np.ndarray) -> float:
    return float(np.count_nonzero(mask == 0)) / mask.size


def _stamp_ball(mask, cz, cy, cx, r):
    nz, ny, nx = mask.shape
    lo = [int(np.floor(c - r)) for c in (cz, cy, cx)]
    hi = [int(np.ceil(c + r)) for c in (cz, cy, cx)]
    zz = np.arange(lo[0], hi[0] + 1)
    yy = np.arange(lo[1], hi[1] + 1)
    xx = np.arange(lo[2], hi[2] + 1)
    d2 = ((zz - cz) ** 2)[:, None, None] + ((yy - cy) ** 2)[None, :, None] + ((xx - cx) ** 2)[None, None, :]
    inside = d2 <= r * r
    iz = (zz % nz)[:, None, None]
    iy = (yy % ny)[None, :, None]
    ix = (xx % nx)[None, None, :]
    flat = ((iz * ny + iy) * nx + ix)[inside]
    if len(zz) > nz or len(yy) > ny or len(xx) > nx:
        # a wrapped ball wider than the box can hit a cell twice; count unique cells
        flat = np.unique(flat)
    view = mask.reshape(-1)
    newly = int(np.count_nonzero(view[flat] == 0))
    view[flat] = 1
    return newly


def overlapping_spheres(shape, target_porosity, radius, seed, max_spheres=10_000_000):
    """Overlapping solid spheres with uniformly random centres (periodic).

    ``shape`` is ``(nx, ny, nz)``; ``radius`` is a number or a ``(lo, hi)``
    range drawn uniformly per sphere.  Spheres are added until the pore
    fraction is <= ``target_porosity``.  Returns a ``(nz, ny, nx)`` uint8 mask.
    """
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    mask = np.zeros((nz, ny, nx), dtype=np.uint8)
    pores = mask.size
    goal = target_porosity * mask.size
    n = 0
    while pores > goal and n < max_spheres:
        cx, cy, cz = rng.uniform(0, nx), rng.uniform(0, ny), rng.uniform(0, nz)
        r = float(radius) if np.isscalar(radius) else float(rng.uniform(radius[0], radius[1]))
        pores -= _stamp_ball(mask, cz, cy, cx, r)
        n += 1
    return mask


def random_cylinders(shape, target_porosity, radius, seed, max_cylinders=1_000_000):
    """Random straight solid cylinders with isotropic axes (periodic box).

    A cell is solid when the distance from its centre to the infinite line
    (through a uniform random point along a uniform random unit direction) is
    <= radius, evaluated for the nearest periodic image of the cell along each
    axis.  Cylinders are added until the pore fraction is <= target.
    """
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    mask = np.zeros((nz, ny, nx), dtype=np.uint8)
    goal = target_porosity * mask.size
    pores = mask.size
    n = 0
    L = np.array([nx, ny, nz], dtype=np.float64)

    def nearest(c, size, p):  # per-axis nearest-image offsets (1-D)
        d = np.arange(size, dtype=np.float64) - p
        return d - size * np.round(d / size)

    while pores > goal and n < max_cylinders:
        p = rng.uniform(0, 1, 3) * L
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        dx = nearest(None, nx, p[0])[None, None, :]
        dy = nearest(None, ny, p[1])[None, :, None]
        dz = nearest(None, nz, p[2])[:, None, None]
        t = (dz * v[2] + dy * v[1]) + dx * v[0]
        d2 = (dz * dz + dy * dy) + dx * dx - t * t
        hit = (d2 <= radius * radius) & (mask == 0)
        pores -= int(np.count_nonzero(hit))
        mask[hit] = 1
        n += 1
    return mask


def blob_phase_field(mask, seed, n_blobs=None, sigma=None, saturation=0.5):
    """Seeded Gaussian-blob field on the pore space, thresholded at the pore
    quantile that gives the requested wetting saturation.  Returns a float64
    array of +1 (wetting) / -1 (non-wetting) on pores and 0 on solids, in the
    mask's (nz, ny, nx) layout."""
    nz, ny, nx = mask.shape
    rng = np.random.default_rng(seed)
    if sigma is None:
        sigma = max(nx, ny, nz) / 16.0
    if n_blobs is None:
        n_blobs = 64
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    field = np.zeros(mask.shape, dtype=np.float64)
    for _ in range(n_blobs):
        c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
        a = rng.choice([-1.0, 1.0])
        dx = x - c[0]
        dy = y - c[1]
        dz = z - c[2]
        dx -= nx * np.round(dx / nx)
        dy -= ny * np.round(dy / ny)
        dz -= nz * np.round(dz / nz)
        field += a * np.exp(-(dx * dx + dy * dy + dz * dz) / (2 * sigma * sigma))
    pore = mask == 0
    thr = np.quantile(field[pore], 1.0 - saturation)
    psi = np.where(field > thr, 1.0, -1.0)
    psi[~pore] = 0.0
    return psi


def write_ascii(path, mask):
    """Reference ASCII geometry: one token per line, x fastest."""
    flat = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    with open(path, "wb") as fh:
        fh.write(_ascii_bytes(flat))


def _ascii_bytes(flat):
    out = np.empty(flat.size * 2, dtype=np.uint8)
    out[0::2] = flat.astype(np.uint8) + ord("0")
    out[1::2] = ord("\n")
    return out.tobytes()


def write_binary(path, mask):
    """Reference binary geometry: int32, C order [i][j][k] (z fastest)."""
    arr = np.ascontiguousarray(np.transpose(mask, (2, 1, 0)).astype(np.int32))
    arr.tofile(path)


def read_ascii(path, shape):
    nx, ny, nz = shape
    toks = np.array(open(path, "rb").read().split(), dtype=np.int64)
    if toks.size < nx * ny * nz:
        raise ValueError(f"{path}: {toks.size} tokens, expected {nx * ny * nz}")
    return (toks[: nx * ny * nz] != 0).astype(np.uint8).reshape(nz, ny, nx)


def read_binary(path, shape):
    nx, ny, nz = shape
    need = nx * ny * nz * 4
    if os.path.getsize(path) < need:
        raise ValueError(f"{path}: shorter than {need} bytes")
    arr = np.fromfile(path, dtype=np.int32, count=nx * ny * nz).reshape(nx, ny, nz)
    return np.ascontiguousarray(np.transpose(arr, (2, 1, 0)) != 0).astype(np.uint8)
