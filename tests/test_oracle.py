"""The oracle is pinned before it is trusted.

* The C restatement (oracle/lbm_oracle.c) must reproduce, bit for bit, the
  golden fixtures produced by the reference solver compiled from its own
  source (tests/golden/make_golden.py), and the compiled reference itself on
  fresh seeded geometries when oracle/_ref is present.
* The closed-form moment expressions the CUDA kernels use (equilibrium
  moments, Guo forcing moments, M^-1 = M^T diag(1/|row|^2)) are checked
  against M f_eq, M G and the Gauss-Jordan inverse computed from the
  reference's definitions.
"""
import numpy as np
import pytest

from helpers import load_golden, spheres


def run_restatement(oracle_mod, mask, nu, g, steps):
    run = oracle_mod.SinglePhaseRun(mask, nu, g)
    run.step(steps)
    return run


def test_restatement_matches_reference_fixture_small(oracle_mod):
    gd = load_golden("sp_small.npz")
    run = oracle_mod.SinglePhaseRun(gd["mask"], float(gd["nu"]), tuple(gd["g"]))
    assert np.array_equal(run.coor, gd["coor"])
    assert np.array_equal(run.nei.reshape(-1, 19), gd["nei_loc"])
    assert np.array_equal(run.MI.reshape(19, 19), gd["MI"])
    run.step(int(gd["steps"]))
    e, umax, umean = run.error()
    pe, perm, uave = run.perm()
    f, u, rho = run.fields()
    assert np.array_equal(f, gd["f"])
    assert np.array_equal(u, gd["u"])
    assert np.array_equal(rho, gd["rho"])
    d = np.array([e, umax, umean, pe, *perm, uave])
    np.testing.assert_array_equal(d, gd["diag"])


def test_restatement_matches_reference_fixture_24(oracle_mod):
    import hashlib

    gd = load_golden("sp_24.npz")
    run = oracle_mod.SinglePhaseRun(gd["mask"], float(gd["nu"]), tuple(gd["g"]))
    assert hashlib.sha256(run.coor.tobytes()).hexdigest() == str(gd["coor_digest"])
    assert hashlib.sha256(run.nei.reshape(-1, 19).tobytes()).hexdigest() == str(gd["nei_digest"])
    run.step(int(gd["steps"]))
    f, u, rho = run.fields()
    assert np.array_equal(u, gd["u"])
    assert np.array_equal(rho, gd["rho"])
    assert hashlib.sha256(f.tobytes()).hexdigest() == str(gd["f_digest"])


@pytest.mark.parametrize("shape,phi,r,seed,g", [
    ((3, 3, 3), 0.7, 0.9, 1, (1e-5, 0.0, 0.0)),        # tiny periodic box, self-wrapping links
    ((17, 9, 6), 0.5, 2.2, 7, (2e-6, 1e-6, 3e-6)),     # ragged sizes, body force on every axis
    ((10, 12, 14), 0.95, 1.5, 3, (1e-4, 0.0, 0.0)),    # nearly empty box
])
def test_restatement_matches_compiled_reference(oracle_mod, shape, phi, r, seed, g):
    if not oracle_mod.reference_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    mask = spheres(shape, phi, r, seed)
    ref = oracle_mod.ReferenceSP3()
    ref.create(mask, 0.12, g, binary=bool(seed % 2))
    run = oracle_mod.SinglePhaseRun(mask, 0.12, g)
    assert np.array_equal(ref.coor(), run.coor)
    assert np.array_equal(ref.nei_loc(), run.nei.reshape(-1, 19))
    for _ in range(3):
        ref.step(7)
        run.step(7)
        fr, ur, rr = ref.fields()
        fo, uo, ro = run.fields()
        assert np.array_equal(fr, fo) and np.array_equal(ur, uo) and np.array_equal(rr, ro)
    assert np.array_equal(np.array(ref.error()), np.array(run.error()))
    er, pr, ar = ref.perm()
    eo, po, ao = run.perm()
    assert np.array_equal(pr, po) and ar == ao


def _feq(rho, u):
    e = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
                  [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1], [1, 0, 1],
                  [-1, 0, 1], [1, 0, -1], [-1, 0, -1]], dtype=np.float64)
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    eu = e @ u
    return w * rho * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * u @ u), e, w


def test_closed_form_moments_used_by_kernels(oracle_mod):
    M, MI = oracle_mod.Restatement().matrices()
    rng = np.random.default_rng(0)
    for _ in range(20):
        rho = 1 + 0.01 * rng.standard_normal()
        u = 0.05 * rng.standard_normal(3)
        g = 1e-3 * rng.standard_normal(3)
        feq, e, w = _feq(rho, u)
        G = w * (3 * ((e - u) @ g) + 9 * (e @ u) * (e @ g))
        meq = M @ feq
        ux, uy, uz = u
        usq = u @ u
        p9 = rho * (2 * ux * ux - uy * uy - uz * uz)
        p11 = rho * (uy * uy - uz * uz)
        closed = np.array([rho, -11 * rho + 19 * rho * usq, 3 * rho - 5.5 * rho * usq, rho * ux, -2 / 3 * rho * ux,
                           rho * uy, -2 / 3 * rho * uy, rho * uz, -2 / 3 * rho * uz, p9, -0.5 * p9, p11, -0.5 * p11,
                           rho * ux * uy, rho * uy * uz, rho * ux * uz, 0, 0, 0])
        np.testing.assert_allclose(meq, closed, rtol=0, atol=1e-14)
        ug = u @ g
        f9 = 2 * (2 * ux * g[0] - uy * g[1] - uz * g[2])
        f11 = 2 * (uy * g[1] - uz * g[2])
        closed_g = np.array([0, 38 * ug, -11 * ug, g[0], -2 / 3 * g[0], g[1], -2 / 3 * g[1], g[2], -2 / 3 * g[2], f9,
                             -0.5 * f9, f11, -0.5 * f11, ux * g[1] + uy * g[0], uy * g[2] + uz * g[1],
                             ux * g[2] + uz * g[0], 0, 0, 0])
        np.testing.assert_allclose(M @ G, closed_g, rtol=0, atol=1e-17)
    # deviation offsets M w used by the deviation-form kernels
    np.testing.assert_allclose(M @ w, [1, -11, 3] + [0] * 16, atol=1e-15)
    # orthogonal rows: M^-1 = M^T diag(1/|row|^2) up to the Gauss-Jordan round-off
    norms = (M * M).sum(axis=1)
    np.testing.assert_allclose(MI, M.T / norms[None, :], rtol=0, atol=1e-15)
    assert list(norms.astype(int)) == [19, 2394, 252, 10, 40, 10, 40, 10, 40, 36, 72, 12, 24, 4, 4, 4, 8, 8, 8]
