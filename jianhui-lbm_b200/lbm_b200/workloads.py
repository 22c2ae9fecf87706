"""Seeded synthetic workloads of the benchmark configurations.

No public dataset exists for these runs; every geometry is generated from a
seed with the sizes and distributions the configurations state:

1. 64^3 overlapping spheres r = 6, porosity 0.40, tau = 1 (nu = 1/6), gx = 1e-6.
2. 256^3 overlapping spheres r ~ U[4,10], porosity 0.35, tau = 0.8, gx = 1e-6.
3. 128^3 random straight cylinders r = 3, porosity 0.6; Gaussian-blob
   wetting field at saturation 0.5.
4. 64 sphere packs: edge log-U[48,160], porosity U[0.25,0.5], r = 5,
   tau = 0.8, gx = 1e-6.
5. a Poisson request stream: edge log-U[32,192], porosity U[0.2,0.5],
   r ~ U[3,8], gx = 1e-6, tau = 0.8.
"""
from __future__ import annotations

import numpy as np

from . import geometry as G

NU_TAU08 = 0.1          # tau = 0.8
NU_TAU1 = 1.0 / 6.0     # tau = 1.0


def config1_mask(seed=2024):
    return G.overlapping_spheres((64, 64, 64), 0.40, 6.0, seed)


def config2_mask(seed=20260101):
    return G.overlapping_spheres((256, 256, 256), 0.35, (4.0, 10.0), seed)


def config3(seed=303):
    mask = G.random_cylinders((128, 128, 128), 0.6, 3.0, seed)
    psi = G.blob_phase_field(mask, seed + 1, saturation=0.5)
    return mask, psi


def _log_uniform(rng, lo, hi):
    return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))


def config4_instances(n=64, seed=404, gx=1e-6):
    """(mask, nu, g) for the batched permeability solves."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        edge = int(round(_log_uniform(rng, 48, 160)))
        phi = float(rng.uniform(0.25, 0.50))
        mask = G.overlapping_spheres((edge, edge, edge), phi, 5.0, int(rng.integers(1 << 31)))
        out.append((mask, NU_TAU08, (gx, 0.0, 0.0)))
    return out


def config5_requests(n=48, seed=505, rate_per_s=2.0, gx=1e-6):
    """[(arrival_time_s, mask, nu, g)] for the serving stream (Poisson arrivals)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        edge = int(round(_log_uniform(rng, 32, 192)))
        phi = float(rng.uniform(0.20, 0.50))
        r = float(rng.uniform(3.0, 8.0))
        mask = G.overlapping_spheres((edge, edge, edge), phi, r, int(rng.integers(1 << 31)))
        out.append((t, mask, NU_TAU08, (gx, 0.0, 0.0)))
    return out
