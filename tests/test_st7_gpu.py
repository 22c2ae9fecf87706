"""D3Q7 solute kernels on the GPU against the restatement, and the
flow -> solute coupling.

FP64: concentration bit-identical to the restatement.  FP32: within 1e-5 of
the maximum concentration.  The velocity file written from a flow solve reads
back in the library's id order exactly.
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


@pytest.fixture(scope="module")
def flow_case(L):
    mask = spheres((26, 22, 18), 0.55, 3.0, seed=61)
    with L.SinglePhase(mask, 0.1, (1e-4, 2e-5, 0.0), precision="f64") as s:
        s.step(300)
        _, u = s.fields()
    rng = np.random.default_rng(3)
    c0 = rng.uniform(0.0, 1.0, mask.shape)
    return mask, u, c0


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_st7_matches_restatement(L, oracle_mod, flow_case, precision):
    mask, u, c0 = flow_case
    ref = oracle_mod.SoluteRun(mask, c0, 0.03, u)
    ref.step(157)
    want = ref.concentration()
    with L.Solute(mask, c0, 0.03, u_nodes=u, precision=precision) as s:
        s.step(100)
        s.step(57)
        got = s.concentration()
    if precision == "f64":
        assert np.array_equal(got, want)
    else:
        assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    assert abs(got[1:].sum() - c0[mask == 0].sum()) <= 1e-4 * c0[mask == 0].sum()


def test_velocity_file_round_trip_and_coupling(L, flow_case, tmp_path):
    mask, _, c0 = flow_case
    with L.SinglePhase(mask, 0.1, (1e-4, 2e-5, 0.0), precision="f64", ordering="hilbert") as s:
        s.step(120)
        _, u = s.fields()
        path = str(tmp_path / "Velocity_for_solute_120.0.bin")
        L.write_velocity_for_solute(s, path)
        raw = np.fromfile(path, dtype=np.float64)
        assert raw.size == 3 * s.count
        back = L.read_velocity_for_solute(path, mask)
        assert np.array_equal(back, u)
        # slab order: the first record is the pore cell with the smallest i*ny*nz + j*nz + k
        coor = s.compaction()
        first = 1 + int(np.argmin(coor[1:]))
        assert np.array_equal(raw[:3], u[first])
        with L.Solute(None, c0, 0.03, flow=s, precision="f64") as a, \
                L.Solute(mask, c0, 0.03, u_nodes=u, precision="f64") as b:
            a.step(40)
            b.step(40)
            assert np.array_equal(a.concentration(), b.concentration())


def test_st7_gpu_matches_the_reference_program(L, tmp_path):
    """FP64 against the solute program itself (two slab ranks, fixture
    st7_slab.npz): the velocity is read from the slab-order record file the
    reference reads, the concentration compared bit for bit at the reference's
    backups (steps 20, 40, 60: 21, 41, 61 updates)."""
    import os

    from helpers import GOLDEN, unpack_mask

    z = np.load(os.path.join(GOLDEN, "st7_slab.npz"))
    mask = unpack_mask(z["mask"], z["shape"])
    path = str(tmp_path / "Velocity_for_solute_100.bin")
    z["u_slab"].tofile(path)  # the two ranks' records, concatenated: the one-rank slab file
    u = L.read_velocity_for_solute(path, mask, order="slab")
    k, j, i = np.nonzero(mask == 0)
    nz, ny, nx = mask.shape
    order = np.argsort(i * ny * nz + j * nz + k, kind="stable")
    with L.Solute(mask, z["c0"].astype(np.float64), float(z["diffusivity"]), u_nodes=u, precision="f64") as s:
        done = -1
        for m in (20, 40, 60):
            s.step(m - done)
            done = m
            want = np.zeros(s.count + 1)
            want[1 + order] = z[f"c{m}"]
            assert np.array_equal(s.concentration()[1:], want[1:]), m
