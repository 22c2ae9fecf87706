"""Pins of the D3Q7 solute restatement by its physics.

The reference solute solver is decomposed in x-slabs and needs two or more
MPI ranks, so it cannot run under the one-rank stand-in; its restatement
(oracle/lbm_oracle_st.c) is checked against properties of the scheme it
implements instead:
  * mass: sum C is conserved with halfway bounce-back and periodic wrap;
  * diffusion: with u = 0 a Gaussian spreads as sigma^2(t) = sigma0^2 + 2 D t,
    D = (tau_s - 1/2)/3;
  * advection: the centroid moves with the imposed uniform velocity.
"""
import numpy as np


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
