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


def test_group_perm_matches_the_slab_program(oracle_mod):
    """Against the slab program itself at two ranks (sp_slab_perm.npz): the
    restatement's group permeabilities after 101 steps, to the 6 significant
    digits the program prints."""
    import os

    import make_golden
    from helpers import GOLDEN, unpack_mask

    z = np.load(os.path.join(GOLDEN, "sp_slab_perm.npz"))
    mask = unpack_mask(z["mask"], z["shape"])
    lines = z["input"].tobytes().decode().splitlines()
    val = lambda i: lines[i].split(":")[0].split()  # noqa: E731
    nu, g, reso = float(val(13)[0]), tuple(float(x) for x in val(6)), float(val(4)[0])
    u0 = tuple(float(x) for x in val(14))
    run = oracle_mod.SinglePhaseRun(mask, nu, g, u_init=u0)
    run.step(int(val(3)[0]) + 1)
    gp = run.group_perm(**make_golden.SLAB_GROUPS)
    k2 = reso * reso * 1000
    sizes, nsub = make_golden.SLAB_GROUPS["size"], make_golden.SLAB_GROUPS["n_sub"]
    row = 0
    for d in range(4):
        rows = gp[row:row + nsub[d] ** 3]
        row += nsub[d] ** 3
        if nsub[d] == 0:
            continue
        for line, r in zip(z[f"Perm_{sizes[d]}.output"].tobytes().decode().splitlines(), rows):
            p, phi = map(float, line.split())
            assert f"{r[0] * k2:.6g} {r[3]:.6g}" == f"{p:.6g} {phi:.6g}", (line, r)


def test_slab_fixture_is_the_slab_programs_output(oracle_mod, tmp_path):
    import os

    import make_golden
    from helpers import GOLDEN

    if not oracle_mod.slab_program("ref_sp_slab"):
        import pytest

        pytest.skip("slab reference program not built")
    z = np.load(os.path.join(GOLDEN, "sp_slab_perm.npz"))
    make_golden.slab_perm_fixture(str(tmp_path / "f.npz"))
    y = np.load(str(tmp_path / "f.npz"))
    timing = ("Elapsed time is", "The expected completion time is")
    for name in (str(n) for n in z["names"]):
        a, b = z[name].tobytes().decode(), y[name].tobytes().decode()
        if name == "Results.txt":
            a, b = ["\n".join(ln for ln in t.splitlines() if not ln.startswith(timing)) for t in (a, b)]
        assert a == b, name
