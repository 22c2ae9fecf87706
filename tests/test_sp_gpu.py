"""Single-phase kernels on the GPU against the oracle, through the C ABI.

Tolerances (relative to the FP64 oracle, on the same seeded inputs):
  FP64 (LBM_PREC_F64)        bit-exact: populations, rho, u, compaction, table
  FP64 fast (deviation, FMA) |du| <= 1e-10 max|u|, permeability 1e-10
  FP32 deviation             |du| <= 1e-4 max|u|, permeability 1e-4
  FP16 scaled deviation      |du| <= 2e-2 max|u|, permeability 1e-2
"""
import hashlib

import numpy as np
import pytest

from helpers import load_golden, spheres

pytestmark = pytest.mark.gpu

ORDERS = ["reference", "morton", "hilbert", "brick"]


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("order", ORDERS)
def test_fp64_bit_exact_vs_reference_fixture(L, order):
    gd = load_golden("sp_small.npz")
    with L.SinglePhase(gd["mask"], float(gd["nu"]), tuple(gd["g"]), precision="f64", ordering=order,
                       block_size=64) as s:
        assert np.array_equal(s.compaction(), gd["coor"])
        assert np.array_equal(s.table(), gd["nei_loc"])
        s.step(int(gd["steps"]))
        assert np.array_equal(s.populations(), gd["f"])
        rho, u = s.fields()
        assert np.array_equal(u, gd["u"]) and np.array_equal(rho, gd["rho"])
        d = s.reduce()
        e, umax, umean, pe, k0, k1, k2, uave = gd["diag"]
        np.testing.assert_allclose([d["u_rel_change"], d["u_max"], d["u_mean_speed"], d["u_ave"]],
                                   [e, umax, umean, uave], rtol=1e-12)
        np.testing.assert_allclose(d["perm"], [k0, k1, k2], rtol=1e-12)


@pytest.mark.parametrize("g", [(1e-5, -2e-6, 3e-6), (0.0, 4e-6, 0.0), (-3e-6, 0.0, 0.0)])
def test_fp64_bit_exact_any_force_direction(L, oracle_mod, g):
    """The FP64 kernel has a specialisation for a force along x only and a
    general one; both reproduce the FP64 restatement of the reference's
    collision (itself pinned to the compiled reference) bit for bit, here
    with solids, a force with every component, one along y (general path)
    and a negative one along x (specialised path)."""
    mask = spheres((22, 18, 20), 0.5, 3.0, seed=33)
    ref = oracle_mod.SinglePhaseRun(mask, 0.1, g)
    ref.step(60)
    f_ref, u_ref, rho_ref = ref.fields()
    for block in (64, 256):
        with L.SinglePhase(mask, 0.1, g, precision="f64", ordering="morton", block_size=block) as s:
            s.step(59)
            s.step(1)
            assert np.array_equal(s.populations(), f_ref), (g, block)
            rho, u = s.fields()
            assert np.array_equal(u, u_ref) and np.array_equal(rho, rho_ref)


def test_fp64_bit_exact_24(L):
    gd = load_golden("sp_24.npz")
    with L.SinglePhase(gd["mask"], float(gd["nu"]), tuple(gd["g"]), precision="f64", ordering="hilbert") as s:
        assert sha(s.compaction()) == str(gd["coor_digest"])
        assert sha(s.table()) == str(gd["nei_digest"])
        s.step(int(gd["steps"]) - 1)
        s.step(1)
        f = s.populations()
        rho, u = s.fields()
        assert sha(f) == str(gd["f_digest"])
        assert np.array_equal(u, gd["u"]) and np.array_equal(rho, gd["rho"])


def test_fp64_bit_exact_config1_full_size(L):
    """64^3 spheres r=6, porosity 0.40, tau=1, gx=1e-6, 5000 steps: the
    reference's f and u digests and its permeability history."""
    try:
        gd = load_golden("sp_cfg1.npz")
    except FileNotFoundError:
        pytest.skip("sp_cfg1.npz not generated")
    with L.SinglePhase(gd["mask"], float(gd["nu"]), tuple(gd["g"]), precision="f64", ordering="hilbert") as s:
        assert s.count == int(gd["count"])
        every = int(gd["every"])
        for row in gd["history"]:
            s.step(every)
            d = s.reduce()
            n, e, umax, umean, pe, k0, k1, k2, uave = row
            assert d["step"] == int(n)
            np.testing.assert_allclose([d["u_rel_change"], d["u_max"], d["u_mean_speed"], d["u_ave"], d["perm"][0]],
                                       [e, umax, umean, uave, k0], rtol=1e-11)
        rho, u = s.fields()
        assert sha(u) == str(gd["u_digest"]) and sha(rho) == str(gd["rho_digest"])
        assert sha(s.populations()) == str(gd["f_digest"])


@pytest.mark.parametrize("precision,tol_u,tol_k", [("f64fast", 1e-10, 1e-10), ("f32", 1e-4, 1e-4), ("f16", 2e-2, 1e-2)])
def test_reduced_precision_within_tolerance(L, oracle_mod, precision, tol_u, tol_k):
    mask = spheres((28, 24, 20), 0.5, 3.5, seed=9)
    nu, g, steps = 0.1, (1e-5, 0.0, 0.0), 400
    ref = oracle_mod.SinglePhaseRun(mask, nu, g)
    ref.step(steps)
    _, u_ref, _ = ref.fields()
    _, k_ref, _ = ref.perm()
    for order in ("reference", "hilbert"):
        with L.SinglePhase(mask, nu, g, precision=precision, ordering=order) as s:
            s.step(steps)
            _, u = s.fields()
            d = s.reduce()
            scale = np.abs(u_ref).max()
            assert np.abs(u - u_ref).max() <= tol_u * scale, (precision, np.abs(u - u_ref).max() / scale)
            assert abs(d["perm"][0] - k_ref[0]) <= tol_k * abs(k_ref[0])


def test_orderings_and_blocks_give_identical_fp32_results(L):
    mask = spheres((40, 36, 32), 0.45, 4.0, seed=21)
    outs = []
    for order in ORDERS:
        for block in (64, 256, 512):
            with L.SinglePhase(mask, 0.1, (1e-6, 0, 0), precision="f32", ordering=order, block_size=block) as s:
                s.step(37)
                outs.append(s.populations())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


@pytest.mark.parametrize("precision", ["f32", "f16", "f64fast"])
def test_compact_pull_table_gives_the_int32_table_results(L, precision):
    """The compact pull table (per-warp base + 16-bit offsets, int32 fallback
    for warps whose sources spread wider) reads the same sources as the int32
    table: populations bit-identical after 41 steps (single steps and graph
    chains), for two orderings.  98 k fluid nodes, so the warps at the
    periodic wraps exceed the offset range and exercise the fallback."""
    mask = spheres((64, 64, 48), 0.5, 3.5, seed=23)
    for order in ("reference", "morton"):
        outs = []
        for mode in (1, 0):
            with L.SinglePhase(mask, 0.1, (1e-6, 2e-7, 0), precision=precision, ordering=order) as s:
                info = s.table_info()
                assert info["compact"] == 0 and info["table_bytes_per_node"] == 72.0
                assert 0.0 < info["wide_fraction"] < 0.05, info
                s.set_table_mode(1)
                info = s.table_info()
                assert abs(info["table_bytes_per_node"] - (36 + 2.25 + 72 * info["wide_fraction"])) < 1e-9
                s.set_table_mode(mode)
                assert s.table_info()["compact"] == mode
                s.step(5)
                s.step(36)
                outs.append((s.populations(), s.reduce()["perm"]))
        assert np.array_equal(outs[0][0], outs[1][0]), order
        assert outs[0][1] == outs[1][1]


def test_compact_pull_table_with_pressure_faces(L):
    """With pressure faces the step kernel covers the interior nodes only; the
    compact table there gives the int32 table's results bit for bit."""
    mask = spheres((40, 36, 32), 0.5, 3.0, seed=29)
    bc = L.Boundary.make(sub_bc=2, in_bc=1, pressure=(1, 1, 0, 0, 0, 0), rho=(1.0, 1.004, 1.0, 1.0, 1.0, 1.0))
    outs = []
    for mode in (1, 0):
        with L.SinglePhase(mask, 0.1, (0.0, 0.0, 0.0), precision="f32", bc=bc) as s:
            s.set_table_mode(mode)
            s.step(40)
            outs.append(s.populations())
    assert np.array_equal(outs[0], outs[1])


def test_set_state_round_trip_and_restart(L):
    mask = spheres((24, 20, 18), 0.5, 3.0, seed=4)
    with L.SinglePhase(mask, 0.1, (1e-5, 0, 0), precision="f64") as a:
        a.step(15)
        f = a.populations()
        rho, u = a.fields()
        a.step(15)
        f_end = a.populations()
    with L.SinglePhase(mask, 0.1, (1e-5, 0, 0), precision="f64", ordering="morton") as b:
        b.set_state(rho, u, f)
        assert np.array_equal(b.populations(), f)
        b.step(15)
        assert np.array_equal(b.populations(), f_end)


def test_autotune_preserves_state(L):
    mask = spheres((32, 32, 32), 0.45, 4.0, seed=8)
    with L.SinglePhase(mask, 0.1, (1e-5, 0, 0), precision="f64") as a:
        a.step(12)
        want = a.populations()
    with L.SinglePhase(mask, 0.1, (1e-5, 0, 0), precision="f64") as b:
        b.step(5)
        r = b.autotune(trial_steps=4)
        assert r["ordering"] in (0, 1, 2, 3) and r["block"] in (64, 128, 256, 512) and r["mlups"] > 0
        b.step(7)
        assert np.array_equal(b.populations(), want)
    with L.SinglePhase(mask, 0.1, (1e-5, 0, 0), precision="f64", ordering="auto") as c:
        c.step(12)
        assert np.array_equal(c.populations(), want)


def test_mass_conservation_and_uniform_acceleration(L, oracle_mod):
    # no solids: the whole fluid accelerates uniformly, u = g (t + 1/2) in exact
    # arithmetic; the reference's own FP64 rounding drifts by ~3e-11 relative
    mask = np.zeros((8, 6, 10), dtype=np.uint8)
    g = (1e-5, -2e-6, 3e-6)
    ref = oracle_mod.SinglePhaseRun(mask, 0.1, g)
    ref.step(100)
    _, u_ref, rho_ref = ref.fields()
    want = np.array(g) * 100.5
    for prec, tol, mtol in (("f64", 1e-10, 1e-12), ("f32", 1e-5, 1e-6)):
        with L.SinglePhase(mask, 0.1, g, precision=prec) as s:
            s.step(100)
            rho, u = s.fields()
            d = s.reduce()
            if prec == "f64":
                assert np.array_equal(u, u_ref) and np.array_equal(rho, rho_ref)
            np.testing.assert_allclose(u[1:], np.broadcast_to(want, u[1:].shape), rtol=tol)
            assert abs(d["mass"] - s.count) <= mtol * s.count


def test_poiseuille_halfway_bounce_back(L):
    """Channel between two solid planes (halfway walls): with the reference's
    s_other = 8(2-s_v)/(8-s_v) the steady profile is the exact parabola
    u(y) = g/(2 nu) (y+1/2)(H-y-1/2) at the lattice nodes."""
    H = 16
    mask = np.zeros((4, H + 2, 3), dtype=np.uint8)
    mask[:, 0, :] = 1
    mask[:, H + 1, :] = 1
    nu, gx = 1.0 / 6.0, 1e-6
    with L.SinglePhase(mask, nu, (gx, 0, 0), precision="f64") as s:
        s.step(20000)
        rho, u = s.fields()
        coor = s.compaction()
    ny, nz = H + 2, 4
    j = (coor[1:] % (ny * nz)) // nz
    y = j - 1 + 0.5
    exact = gx / (2 * nu) * y * (H - y)
    np.testing.assert_allclose(u[1:, 0], exact, rtol=1e-6)
    assert np.abs(u[1:, 1:]).max() < 1e-14


def elliptic_fibre_mask():
    """The periodic array of elliptic fibres of Accessories/Fibrous_generation.m
    (lines 1-29): 150 x 120 x 3 cells, semi-axes 71.5 (x) and 58.5 (y), centre
    ((lx+1)/2, (ly+1)/2) in 1-based cell indices; neighbours nearly touch
    across the periodic y boundary.  [nz][ny][nx], 1 = solid."""
    lx, ly, lz = 150, 120, 3
    la, lb = 143 / 2, 117 / 2
    ci, cj = (lx + 1) / 2, (ly + 1) / 2
    i = np.arange(1, lx + 1)[None, :]
    j = np.arange(1, ly + 1)[:, None]
    fibre = (j - cj) ** 2 / lb ** 2 + (i - ci) ** 2 / la ** 2 <= 1
    return np.broadcast_to(fibre, (lz, ly, lx)).astype(np.uint8).copy()


def test_elliptic_fibre_array_matches_lubrication(L):
    """Flow along x through the gaps between the fibres.  The reference's
    lubrication estimate (Fibrous_generation.m:42-58) is
    K = 2 lx / (ly * integral of 3 / h(x)^3 dx), h the half gap; the script
    evaluates it on the continuous ellipse (0.148 lu^2 once its printed
    K / (a b) is multiplied back).  Evaluated on the gaps the cell mask
    actually leaves (h = pore cells of column x / 2, unit steps) it is
    0.21138 lu^2, and the converged FP64 permeability agrees within 0.2%
    (the FP64 restatement of the reference gives 0.211308)."""
    mask = elliptic_fibre_mask()
    lx, ly = mask.shape[2], mask.shape[1]
    h = (mask[0] == 0).sum(axis=0) / 2.0
    k_lub = 2 * lx / ly / np.sum(3 / h ** 3)
    assert abs(k_lub - 0.21138) < 1e-4
    with L.SinglePhase(mask, 1.0 / 6.0, (1e-6, 0, 0), precision="f64") as s:
        d = s.run_to_convergence(tol=1e-10, check_every=1000, max_steps=60000)
    assert d["status"] == 0
    assert abs(d["perm"][0] - k_lub) <= 2e-3 * k_lub, (d["perm"][0], k_lub)
    assert abs(d["perm"][0] - 0.2113083) <= 1e-6


def test_run_to_convergence_matches_oracle_rule(L, oracle_mod):
    mask = spheres((24, 24, 24), 0.5, 3.0, seed=30)
    nu, g, tol, every = 0.1, (1e-5, 0, 0), 1e-4, 50
    ref = oracle_mod.SinglePhaseRun(mask, nu, g)
    prev, n_ref = 0.0, None
    for it in range(1, 200):
        ref.step(every)
        _, _, uave = ref.perm()
        if prev and abs((prev - uave) / prev) < tol:
            n_ref = it * every
            break
        prev = uave
    assert n_ref is not None
    with L.SinglePhase(mask, nu, g, precision="f64") as s:
        d = s.run_to_convergence(tol=tol, check_every=every, max_steps=10000)
        assert d["converged"] == 1 and d["step"] == n_ref
    with L.SinglePhase(mask, nu, g, precision="f32") as s:
        d = s.run_to_convergence(tol=tol, check_every=every, max_steps=10000)
        assert d["converged"] == 1 and abs(d["step"] - n_ref) <= every
    with L.SinglePhase(mask, nu, g, precision="f32") as s:
        d = s.run_to_convergence(tol=1e-12, check_every=every, max_steps=200)
        assert d["status"] == -6 and d["step"] == 200


def test_create_from_input_file(L, tmp_path):
    from lbm_b200 import geometry as G

    mask = spheres((24, 20, 16), 0.5, 3.0, seed=12)
    G.write_ascii(tmp_path / "mask_24.dat", mask)
    txt = open(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "INPUT_sp.dat")).read()
    txt = txt.replace("mask_24.dat", str(tmp_path / "mask_24.dat"))
    (tmp_path / "INPUT.dat").write_text(txt)
    s = L.SinglePhase.from_input(str(tmp_path / "INPUT.dat"), precision="f64")
    try:
        assert s.count == int((mask == 0).sum())
        s.step(3)
        rho, u = s.fields()
        assert np.isfinite(u).all()
    finally:
        s.close()


def test_errors_are_reported_not_fatal(L):
    with pytest.raises(L.LbmError) as e:
        L.SinglePhase(np.ones((4, 4, 4), dtype=np.uint8), 0.1)
    assert e.value.status == -1
    # a diverging run is stopped by the reference's NaN rule
    mask = np.zeros((6, 6, 6), dtype=np.uint8)
    with L.SinglePhase(mask, 0.1, (5.0, 0, 0), precision="f64") as s:
        with pytest.raises(L.LbmError) as e:
            s.run_to_convergence(tol=1e-9, check_every=20, max_steps=2000)
        assert e.value.status in (-5, -9)
