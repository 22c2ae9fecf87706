"""Pins of the colour-gradient oracle: the C restatement
(oracle/lbm_oracle_cg.c) reproduces bit for bit the fixture produced by the
reference colour-gradient solver compiled from its own source, and the
compiled reference itself on a fresh seeded case."""
import numpy as np
import pytest

from helpers import load_golden


def args_of(gd):
    a = gd["args"]
    return dict(nu_l=a[0], nu_g=a[1], psi_solid=a[2], cap_a=a[3], g=(a[4], a[5], a[6]),
                body_force_phase=int(a[7]), flux_psi=a[8], flux_umax=a[9])


def test_cg_restatement_matches_reference_fixture(oracle_mod):
    gd = load_golden("cg_small.npz")
    run = oracle_mod.ColourGradientRun(gd["mask"], gd["psi0"], **args_of(gd))
    assert np.array_equal(run.coor, gd["coor"])
    assert np.array_equal(run.nei.reshape(-1, 19), gd["nei_loc"])
    run.step(int(gd["steps"]))
    d = run.fields()
    for k in ("f", "u", "rho", "psi", "rho_r", "rho_b"):
        assert np.array_equal(d[k], gd[k]), k
    e, pl, pg, ua = run.perm()
    assert np.array_equal(pl, gd["perm_l"]) and np.array_equal(pg, gd["perm_g"]) and ua == gd["u_ave"]
    assert run.saturation() == gd["saturation"]


def test_cg_restatement_matches_compiled_reference(oracle_mod):
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built")
    from lbm_b200 import geometry as G

    mask = G.random_cylinders((13, 11, 9), 0.55, 1.8, seed=8)
    psi = G.blob_phase_field(mask, seed=9, saturation=0.4)
    kw = dict(nu_l=0.12, nu_g=0.05, psi_solid=-0.3, cap_a=5e-3, g=(2e-5, -1e-5, 0.0), body_force_phase=1,
              flux_psi=0.9, flux_umax=0.05)
    ref = oracle_mod.ReferenceCG3()
    ref.create(mask, psi, **kw)
    run = oracle_mod.ColourGradientRun(mask, psi, **kw)
    M, MI = ref.matrices()
    assert np.array_equal(M, run.M.reshape(19, 19)) and np.array_equal(MI, run.MI.reshape(19, 19))
    for _ in range(3):
        ref.step(9)
        run.step(9)
        a, b = ref.fields(), run.fields()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    assert ref.saturation() == run.saturation()


def test_cg_guo_moment_closed_forms(oracle_mod):
    """The FP32 colour-gradient kernel uses M G in closed form for the CG
    basis: nine non-zero rows.  Checked against M times the reference's Guo
    term G_q = w_q [3 (e_q - u).g + 9 (e_q.u)(e_q.g)] (CG3:2745-2825)."""
    from lbm_b200 import geometry as G

    mask = G.random_cylinders((8, 8, 8), 0.6, 1.5, seed=1)
    run = oracle_mod.ColourGradientRun(mask, G.blob_phase_field(mask, seed=2, saturation=0.5), nu_l=0.1, nu_g=0.1,
                                       psi_solid=0.7, cap_a=1e-3, g=(1e-5, 0.0, 0.0))
    M = run.M.reshape(19, 19)
    # CG velocity order (CG3:188-196): the columns of M are polynomials of e
    e = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
                  [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1], [0, 1, 1],
                  [0, -1, -1], [0, 1, -1], [0, -1, 1]], dtype=float)
    assert np.array_equal(M[3], e[:, 0]) and np.array_equal(M[5], e[:, 1]) and np.array_equal(M[7], e[:, 2])
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    rng = np.random.default_rng(5)
    for _ in range(5):
        u, g = rng.normal(size=3) * 0.05, rng.normal(size=3) * 1e-4
        Gq = w * (3 * ((e - u) @ g) + 9 * (e @ u) * (e @ g))
        mg = M @ Gq
        xx, yy, zz = u * g
        want = np.zeros(19)
        want[1] = 2 * (xx + yy + zz)
        want[3], want[5], want[7] = g
        want[9] = 4 * xx - 2 * yy - 2 * zz
        want[11] = 2 * yy - 2 * zz
        want[13] = u[0] * g[1] + u[1] * g[0]
        want[14] = u[1] * g[2] + u[2] * g[1]
        want[15] = u[0] * g[2] + u[2] * g[0]
        assert np.allclose(mg, want, rtol=0, atol=1e-18)
