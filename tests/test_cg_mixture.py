"""Mixture injection of the colour-gradient program (mix_psi_thickness > 0).

The initial phase is built from the geometry by psi_mixture_ini
(CG3:6151-6350) instead of being read from the phase file.  The library's
host port (lbm_cg_mixture_phase) is compared, cell by cell at every fluid
node, with the phase the reference program itself builds: the compiled
reference (oracle/_ref/libref_cg3.so) runs its own geometry set-up and init
with the mixture settings, and its initial psi is read back.  Geometries with
ny = nz (the reference reads outside the plane otherwise).  The GPU half --
the zero-surface-tension layer in the collision and the whole program's
files -- is tests/test_cg_outputs_gpu.py (cg_outputs_mix.npz)."""
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


@pytest.mark.parametrize("shape,phi,seed,thickness,portion", [
    ((16, 12, 12), 0.6, 31, 3, 0.6), ((20, 16, 16), 0.5, 5, 4, 0.5), ((18, 14, 14), 0.7, 8, 2, 0.9),
    ((24, 20, 20), 0.55, 3, 6, 0.3)])
def test_mixture_phase_equals_the_reference_initialisation(L, oracle_mod, shape, phi, seed, thickness, portion):
    from lbm_b200 import geometry as G

    if not os.path.exists(os.path.join(os.path.dirname(oracle_mod.__file__), "_ref", "libref_cg3.so")):
        pytest.skip("reference colour-gradient library not built")
    mask = G.overlapping_spheres(shape, phi, 2.5, seed)
    ref = oracle_mod.ReferenceCG3()
    ref.set_mixture(thickness, portion)
    # the reference reports the wetting share on stdout
    out = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    try:
        n = ref.create(mask, np.ones(mask.shape), 0.1, 0.1, 0.7, 1e-3, (1e-5, 0.0, 0.0))
    finally:
        os.dup2(out, 1)
        os.close(null)
        os.close(out)
        ref.set_mixture(0, 0.5)
    rho, psi, rr, rb = (np.zeros(n + 1) for _ in range(4))
    ref.L.ref_cg3_get_scalars(rho, psi, rr, rb)
    coor = np.zeros(n + 1, dtype=np.int32)
    ref.L.ref_cg3_get_coor(coor)
    mine = L.mixture_phase(mask, thickness, portion)
    nz, ny, nx = mask.shape
    c = coor[1:]
    i, j, k = c // (ny * nz), (c % (ny * nz)) // nz, c % nz
    assert np.array_equal(mine[k, j, i], psi[1:])
    assert (mine < 0).any() and (mine > 0).any()
    # only the buffer x <= thickness holds component B
    assert (mine[:, :, thickness + 1:] == 1).all()


def test_mixture_phase_rejects_a_buffer_outside_the_box(L):
    mask = np.zeros((8, 8, 10), dtype=np.uint8)
    for bad in (0, 10, 12):
        with pytest.raises(L.LbmError):
            L.mixture_phase(mask, bad, 0.5)
