"""Pins of the D3Q7 solute restatement (oracle/lbm_oracle_st.c).

Against the reference program itself: the solute program is decomposed in
x-slabs and needs two or more MPI ranks; tests/golden/st7_slab.npz was made
by running it (and the slab single-phase program for its velocity field) as
two processes under the multi-process MPI stand-in (make_golden.py --st7).
The restatement must reproduce its concentration bit for bit.  Also against
properties of the scheme:
  * mass: sum C is conserved with halfway bounce-back and periodic wrap;
  * diffusion: with u = 0 a Gaussian spreads as sigma^2(t) = sigma0^2 + 2 D t,
    D = (tau_s - 1/2)/3;
  * advection: the centroid moves with the imposed uniform velocity.
"""
import os

import numpy as np
import pytest

from helpers import GOLDEN, unpack_mask


def gaussian(shape, centre, sigma):
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r2 = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2
    return np.exp(-r2 / (2 * sigma * sigma))


def test_st7_conserves_mass_with_walls(oracle_mod):
    from lbm_b200 import geometry as G

    mask = G.overlapping_spheres((20, 18, 16), 0.6, 3.0, seed=5)
    n = int((mask == 0).sum())
    rng = np.random.default_rng(0)
    u = np.zeros((n + 1, 3))
    u[1:] = 0.02 * rng.standard_normal((n, 3))
    c0 = rng.uniform(0, 1, mask.shape)
    run = oracle_mod.SoluteRun(mask, c0, 0.05, u)
    m0 = run.concentration()[1:].sum()
    run.step(200)
    assert abs(run.concentration()[1:].sum() - m0) <= 1e-11 * m0


def test_st7_diffusion_variance_grows_as_2Dt(oracle_mod):
    shape, D, steps = (64, 9, 9), 0.05, 300
    mask = np.zeros((shape[2], shape[1], shape[0]), dtype=np.uint8)
    c0 = np.broadcast_to(gaussian((shape[0], 1, 1), (31.5, 0, 0), 2.0), mask.shape).copy()
    n = mask.size
    run = oracle_mod.SoluteRun(mask, c0, D, np.zeros((n + 1, 3)))
    run.step(steps)
    c = run.concentration()[1:].reshape(mask.shape)[0, 0]
    x = np.arange(shape[0])
    var = ((x - 31.5) ** 2 * c).sum() / c.sum()
    want = 4.0 + 2 * D * steps
    assert abs(var - want) <= 0.01 * want


def test_st7_centroid_moves_with_the_flow(oracle_mod):
    shape, steps, ux = (80, 6, 6), 200, 0.05
    mask = np.zeros((shape[2], shape[1], shape[0]), dtype=np.uint8)
    c0 = np.broadcast_to(gaussian((shape[0], 1, 1), (20.0, 0, 0), 3.0), mask.shape).copy()
    n = mask.size
    u = np.zeros((n + 1, 3))
    u[1:, 0] = ux
    run = oracle_mod.SoluteRun(mask, c0, 0.02, u)
    run.step(steps)
    c = run.concentration()[1:].reshape(mask.shape)[0, 0]
    x = np.arange(shape[0])
    centroid = (x * c).sum() / c.sum()
    assert abs(centroid - (20.0 + ux * steps)) <= 0.05


def slab_permutation(mask):
    """Position of each pore cell of the x-fastest compaction in the slab
    programs' order (x outer, z fastest; ranks own consecutive x ranges, so
    their records concatenate to this order)."""
    nz, ny, nx = mask.shape
    k, j, i = np.nonzero(mask == 0)
    return np.argsort(i * ny * nz + j * nz + k, kind="stable")


def st7_case():
    z = np.load(os.path.join(GOLDEN, "st7_slab.npz"))
    mask = unpack_mask(z["mask"], z["shape"])
    order = slab_permutation(mask)
    n = order.size
    u = np.zeros((n + 1, 3))
    u[1 + order] = z["u_slab"].reshape(-1, 3)
    want = {}
    for m in z["steps"]:
        c = np.zeros(n + 1)
        c[1 + order] = z[f"c{int(m)}"]
        want[int(m)] = c
    return z, mask, u, want


def test_st7_matches_the_reference_program(oracle_mod):
    z, mask, u, want = st7_case()
    run = oracle_mod.SoluteRun(mask, z["c0"].astype(np.float64), float(z["diffusivity"]), u)
    done = -1
    for m in sorted(want):
        run.step(m - done)  # the reference runs steps n = 0..m before its step-m backup
        done = m
        assert np.array_equal(run.concentration()[1:], want[m][1:]), m


def test_st7_fixture_is_the_reference_programs_output(oracle_mod, tmp_path):
    """Re-runs the two slab programs (where they were built) and compares
    with the fixture."""
    import make_golden

    if not (oracle_mod.slab_program("ref_sp_slab") and oracle_mod.slab_program("ref_st7_slab")):
        pytest.skip("slab reference programs not built")
    if not os.path.isdir(oracle_mod.REFERENCE_ROOT):
        pytest.skip("reference sample INPUT not present")
    z = np.load(os.path.join(GOLDEN, "st7_slab.npz"))
    make_golden.st7_fixture(str(tmp_path / "st7_slab.npz"))
    y = np.load(str(tmp_path / "st7_slab.npz"))
    for k in ("u_slab", "rank_nodes", "c20", "c40", "c60", "c0"):
        assert np.array_equal(y[k], z[k]), k
