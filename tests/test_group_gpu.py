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


def test_slab_program_sub_volume_permeabilities(L, tmp_path):
    """Against the slab single-phase program itself, run at two ranks
    (fixture sp_slab_perm.npz): its Perm_<size>.output files (Comput_Grop_Perm)
    and the LOCAL permeability of its Results.txt (Comput_Perm_LOCAL) after 101
    steps, printed with 6 significant digits, from lbm_group_perm /
    lbm_local_perm on the FP64 state of the same INPUT file."""
    import os

    import make_golden
    from helpers import GOLDEN, unpack_mask
    from lbm_b200 import geometry as G

    z = np.load(os.path.join(GOLDEN, "sp_slab_perm.npz"))
    mask = unpack_mask(z["mask"], z["shape"])
    G.write_ascii(str(tmp_path / "mask.dat"), mask)
    lines = z["input"].tobytes().decode().splitlines()
    lines[1] = f"{tmp_path / 'mask.dat'}\t\t:{lines[1].split(':', 1)[1]}"
    (tmp_path / "INPUT.dat").write_text("\n".join(lines) + "\n")
    s = L.SinglePhase.from_input(str(tmp_path / "INPUT.dat"), precision="f64")
    try:
        reso2k = s.input["reso"] ** 2 * 1000
        s.step(s.input["n_max"] + 1)
        gp = s.group_perm(**make_golden.SLAB_GROUPS)
        local = s.local_perm() * reso2k
    finally:
        s.close()

    def close(got, want):
        return abs(got - want) <= 5e-6 * abs(want) + 1e-9

    sizes = make_golden.SLAB_GROUPS["size"]
    nsub = make_golden.SLAB_GROUPS["n_sub"]
    row = 0
    for d in range(4):
        rows = gp[row:row + nsub[d] ** 3]
        row += nsub[d] ** 3
        if nsub[d] == 0:
            continue
        want = [list(map(float, ln.split())) for ln in z[f"Perm_{sizes[d]}.output"].tobytes().decode().splitlines()]
        assert len(want) == len(rows)
        for (p, phi), r in zip(want, rows):
            assert close(r[0] * reso2k, p) and close(r[3], phi), (d, p, phi, r)
    results = z["Results.txt"].tobytes().decode().split("The100th computation result:")[1]
    vals = [float(x) for x in results.split("The LOCAL permiability is:")[1].splitlines()[0].split(",")]
    assert all(close(a, b) for a, b in zip(local, vals)), (local, vals)
