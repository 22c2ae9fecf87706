"""D3Q19 solute program (Single_Phase_3D/Solute_Transport_MPI_Software_Spars.cpp,
"ST19") on the GPU: the solute handle with 19 directions
(lbm_st19_create) and the lbm_st7 driver with --lattice 19.

The reference is the program itself at two slab ranks (the multi-process MPI
stand-in, oracle/_ref/ref_st19_slab), on the inputs of the D3Q7 fixtures:
  st19_slab.npz             concentration at its backups (steps 20, 40, 60);
  st19_outputs.npz          every file of a 61-step run (reports every 20,
                            velocity VTK every 40, concentration VTK every 20,
                            checkpoints every 40);
  st19_outputs_restart.npz  the run restarted from the step-40 checkpoint;
  st19_outputs_lat.npz      a run with a self-defined lattice velocity
                            (dx = 1, dt = 2) and dispersion statistics.
FP64: bit for bit / byte for byte.  FP32: concentration within 1e-5 of the
FP64 fixture after 61 steps.
"""
import hashlib
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN, unpack_mask

pytestmark = pytest.mark.gpu

TIMING = (b"Elapsed time is", b"The expected completion time is")


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def slab_case(L, tmp_path):
    z = np.load(os.path.join(GOLDEN, "st19_slab.npz"))
    mask = unpack_mask(z["mask"], z["shape"])
    path = str(tmp_path / "Velocity_for_solute_100.bin")
    z["u_slab"].tofile(path)  # the two ranks' records, concatenated: the one-rank slab file
    u = L.read_velocity_for_solute(path, mask, order="slab")
    k, j, i = np.nonzero(mask == 0)
    nz, ny, nx = mask.shape
    order = np.argsort(i * ny * nz + j * nz + k, kind="stable")
    return z, mask, u, order


def test_st19_gpu_matches_the_reference_program(L, tmp_path):
    z, mask, u, order = slab_case(L, tmp_path)
    with L.Solute(mask, z["c0"].astype(np.float64), float(z["diffusivity"]), u_nodes=u, precision="f64",
                  lattice=19) as s:
        assert s.directions == 19
        done = -1
        for m in (20, 40, 60):
            s.step(m - done)
            done = m
            want = np.zeros(s.count + 1)
            want[1 + order] = z[f"c{m}"]
            assert np.array_equal(s.concentration()[1:], want[1:]), m


def test_st19_fp32_and_state_round_trip(L, tmp_path):
    z, mask, u, order = slab_case(L, tmp_path)
    c0 = z["c0"].astype(np.float64)
    D = float(z["diffusivity"])
    with L.Solute(mask, c0, D, u_nodes=u, precision="f32", lattice=19) as s:
        s.step(61)
        got = s.concentration()
    want = np.zeros_like(got)
    want[1 + order] = z["c60"]
    assert np.abs(got[1:] - want[1:]).max() <= 1e-5 * np.abs(want).max()
    # populations out in the program's 19-column order and back in: the
    # continued run equals the uninterrupted one
    with L.Solute(mask, c0, D, u_nodes=u, precision="f64", lattice=19) as a, \
            L.Solute(mask, c0, D, u_nodes=u, precision="f64", lattice=19) as b:
        a.step(30)
        g = a.populations()
        c = a.concentration()
        assert g.shape == (a.count + 1, 19)
        a.step(31)
        b.set_state(g, c)
        b.step(31)
        assert np.array_equal(a.concentration(), b.concentration())


def prepare(workdir, golden):
    from lbm_b200 import geometry as G

    shape = tuple(int(s) for s in golden["shape"])
    mask = np.unpackbits(golden["mask"])[: np.prod(shape)].reshape(shape)
    G.write_ascii(os.path.join(workdir, "mask.dat"), mask)
    (workdir / "phase.dat").write_bytes(golden["phase"].tobytes())
    for name in golden["velocity_files"]:
        (workdir / str(name)).write_bytes(golden["file:" + str(name)].tobytes())
    (workdir / "INPUT_st.dat").write_bytes(golden["input"].tobytes())


def run_driver(L, workdir, *args):
    r = subprocess.run([L.driver_path("lbm_st7"), "INPUT_st.dat", "./", "--ranks", "2", "--lattice", "19", *args],
                       cwd=workdir, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def compare(tmp_path, golden, prefix):
    names = [str(n) for n in golden["names"]]
    written = sorted(n[len(prefix):] for n in os.listdir(tmp_path) if n.startswith(prefix))
    assert written == sorted(names)
    for name in names:
        path = tmp_path / (prefix + name)
        if name.startswith("LBM_checkpoint_"):
            width = {"psi": 1, "fg": 19}[name.split("_")[2]]
            a = np.fromfile(path, dtype=np.float64).reshape(-1, width)
            assert hashlib.sha256(np.ascontiguousarray(a[1:]).tobytes()).hexdigest() == str(golden[name]), name
        elif name.startswith("Results"):
            strip = lambda d: b"\n".join(l for l in d.split(b"\n") if not l.startswith(TIMING))
            assert strip(path.read_bytes()) == strip(golden[name].tobytes()), name
        else:
            assert path.read_bytes() == golden[name].tobytes(), name


def test_st19_driver_writes_the_reference_files(L, tmp_path):
    golden = np.load(os.path.join(GOLDEN, "st19_outputs.npz"))
    prepare(tmp_path, golden)
    run_driver(L, tmp_path)
    compare(tmp_path, golden, "st_")


def test_st19_driver_with_lattice_velocity(L, tmp_path):
    """lattice_v with dx = 1, dt = 2: tau_s from c_s^2 = (dx/dt)^2 / 3 and the
    equilibrium's divisions by c2, c4 (ST19:1259-1268, 1480), the reports'
    Peclet and Courant numbers and the dispersion statistics in dx, dt."""
    golden = np.load(os.path.join(GOLDEN, "st19_outputs_lat.npz"))
    prepare(tmp_path, golden)
    run_driver(L, tmp_path)
    compare(tmp_path, golden, "sl_")


def test_st19_driver_restart_matches_the_reference_restart(L, tmp_path):
    first = np.load(os.path.join(GOLDEN, "st19_outputs.npz"))
    prepare(tmp_path, first)
    run_driver(L, tmp_path)
    for r in range(2):
        for what in ("psi", "fg"):
            shutil.copy(tmp_path / f"st_LBM_checkpoint_{what}_40.{r}.bin_input",
                        tmp_path / f"LBM_checkpoint_{what}_40.{r}.bin_input")
    rst = np.load(os.path.join(GOLDEN, "st19_outputs_restart.npz"))
    (tmp_path / "INPUT_st.dat").write_bytes(rst["input"].tobytes())
    run_driver(L, tmp_path)
    compare(tmp_path, rst, "rs_")
