"""Pins of the group-permeability restatement (orc_sp_group_perm,
Comput_Grop_Perm SP:4886-5091).

The slab program that calls Comput_Grop_Perm cannot run at one rank, so the
restatement is pinned through the reference's own Comput_Perm: one cube
covering a cubic box is Comput_Perm's whole-box permeability, bit for bit
(same sums in the same node order, same formula), and that is pinned to the
compiled reference by sp_small / sp_24.  Cubes that tile the box add up to the
whole-box flux and porosity.
"""
import numpy as np


def test_one_cube_is_comput_perm(oracle_mod):
    from lbm_b200 import geometry as G

    mask = G.overlapping_spheres((12, 12, 12), 0.6, 2.5, seed=3)
    run = oracle_mod.SinglePhaseRun(mask, 0.1, (1e-5, 2e-6, -3e-6))
    run.step(30)
    g = run.group_perm([1], [12], [0, 0, 0])
    _, perm, _ = run.perm(1)
    assert np.array_equal(g[0, :3], perm)
    assert g[0, 3] == run.porosity


def test_cubes_tile_the_box(oracle_mod):
    from lbm_b200 import geometry as G

    mask = G.overlapping_spheres((12, 12, 12), 0.6, 2.5, seed=4)
    run = oracle_mod.SinglePhaseRun(mask, 0.1, (1e-5, 0.0, 0.0))
    run.step(25)
    whole = run.group_perm([1], [12], [0, 0, 0])[0]
    parts = run.group_perm([2, 3], [6, 4], [0, 0, 0, 0, 0, 0])
    assert parts.shape == (8 + 27, 4)
    for sl, k in ((slice(0, 8), 8), (slice(8, 35), 27)):
        # perm_d of a cube is Q_cube / size^3 * nu / g: the mean over a tiling is the whole-box value
        assert np.isclose(parts[sl, 0].mean(), whole[0], rtol=1e-12)
        assert np.isclose(parts[sl, 3].mean(), whole[3], rtol=1e-12)
