"""Sub-volume permeabilities on the GPU (lbm_box_sums, lbm_group_perm,
lbm_local_perm) against the restatement.

FP64 state (bit-identical to the restatement), sums in the device's fixed
order: within 1e-12 relative of the restatement's sequential sums.
"""
import numpy as np
import pytest

from helpers import spheres

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def test_group_and_local_perm(L, oracle_mod):
    mask = spheres((24, 20, 16), 0.55, 3.0, seed=17)
    g = (1e-5, 2e-6, 1e-6)
    ref = oracle_mod.SinglePhaseRun(mask, 0.1, g)
    ref.step(120)
    n_sub, size, corner = [1, 2, 3], [16, 8, 5], [0, 0, 0, 4, 2, 0, 1, 3, 0]
    want = ref.group_perm(n_sub, size, corner)
    with L.SinglePhase(mask, 0.1, g, precision="f64", ordering="hilbert") as s:
        s.step(120)
        got = s.group_perm(n_sub, size, corner)
        # local permeability: flux through the plane x = nx - 2 over the cross-sections
        _, u = s.fields()
        coor = s.compaction()
        ny, nz = 20, 16
        ii = coor[1:] // (ny * nz)
        q = u[1:][ii == 24 - 2].sum(axis=0)
        local = s.local_perm()
        # a box reaching outside the grid is clipped; an empty one sums to zero
        b = s.box_sums([(0, 23, 0, 19, 0, 15), (20, 40, -5, 3, 10, 10), (30, 40, 0, 5, 0, 5)])
    assert got.shape == want.shape
    assert np.allclose(got, want, rtol=1e-12, atol=1e-300)
    area = np.array([20 * 16, 24 * 16, 24 * 20])
    assert np.allclose(local, q / area * 0.1 / np.array(g), rtol=1e-12)
    assert np.allclose(b[0, :3], u[1:].sum(axis=0), rtol=1e-12)
    assert b[0, 3] == s.count
    i, j, k = coor[1:] // (ny * nz), (coor[1:] % (ny * nz)) // nz, coor[1:] % nz
    sel = (i >= 20) & (j <= 3) & (k == 10)
    assert np.allclose(b[1, :3], u[1:][sel].sum(axis=0), rtol=1e-12, atol=1e-300)
    assert b[1, 3] == sel.sum()
    assert np.array_equal(b[2], np.zeros(4))
