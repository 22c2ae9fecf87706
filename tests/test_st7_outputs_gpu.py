"""The lbm_st7 driver against the solute program's own output files.

tests/golden/st7_outputs*.npz hold every file the reference solute program
wrote at two ranks from the flow the slab single-phase program made
(Velocity_for_solute_100.<rank>.bin, stored with them): reports every 20
steps, velocity VTK every 40, concentration VTK every 20 and per-rank
checkpoints every 40 in both output layouts (Out_Mode 1 and 0), the
dispersion statistics along x and along z, a self-defined lattice velocity
(lattice_v, dx = 1, dt = 2; st7_outputs_lat.npz), and a restart from the
step-40 checkpoint.  The driver, run on the same files with
--ranks 2 at FP64, must write the same files: text and VTK byte for byte
except the wall-clock lines, the per-rank checkpoints bit for bit (rows 1..).
"""
import hashlib
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN

pytestmark = pytest.mark.gpu

TIMING = (b"Elapsed time is", b"The expected completion time is")


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


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
    r = subprocess.run([L.driver_path("lbm_st7"), "INPUT_st.dat", "./", "--ranks", "2", *args], cwd=workdir,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def strip_timing(data):
    return b"\n".join(l for l in data.split(b"\n") if not l.startswith(TIMING))


def compare(tmp_path, golden, prefix):
    names = [str(n) for n in golden["names"]]
    written = sorted(n[len(prefix):] for n in os.listdir(tmp_path) if n.startswith(prefix))
    assert written == sorted(names)
    for name in names:
        path = tmp_path / (prefix + name)
        if name.startswith("LBM_checkpoint_"):
            width = {"psi": 1, "fg": 7}[name.split("_")[2]]
            a = np.fromfile(path, dtype=np.float64).reshape(-1, width)
            assert hashlib.sha256(np.ascontiguousarray(a[1:]).tobytes()).hexdigest() == str(golden[name]), name
        elif name.startswith("Results"):
            assert strip_timing(path.read_bytes()) == strip_timing(golden[name].tobytes()), name
        else:
            assert path.read_bytes() == golden[name].tobytes(), name


@pytest.mark.parametrize("fixture,prefix", [("st7_outputs.npz", "st_"), ("st7_outputs_b.npz", "sb_"),
                                            ("st7_outputs_dis.npz", "sd_"), ("st7_outputs_dis3.npz", "sz_"),
                                            ("st7_outputs_lat.npz", "sl_")])
def test_st7_driver_writes_the_reference_files(L, fixture, prefix, tmp_path):
    golden = np.load(os.path.join(GOLDEN, fixture))
    prepare(tmp_path, golden)
    run_driver(L, tmp_path)
    compare(tmp_path, golden, prefix)


def test_st7_driver_restart_matches_the_reference_restart(L, tmp_path):
    first = np.load(os.path.join(GOLDEN, "st7_outputs.npz"))
    prepare(tmp_path, first)
    run_driver(L, tmp_path)
    for r in range(2):
        for what in ("psi", "fg"):
            shutil.copy(tmp_path / f"st_LBM_checkpoint_{what}_40.{r}.bin_input",
                        tmp_path / f"LBM_checkpoint_{what}_40.{r}.bin_input")
    rst = np.load(os.path.join(GOLDEN, "st7_outputs_restart.npz"))
    (tmp_path / "INPUT_st.dat").write_bytes(rst["input"].tobytes())
    run_driver(L, tmp_path)
    compare(tmp_path, rst, "rs_")


def test_st7_driver_f32_concentration_close(L, tmp_path):
    golden = np.load(os.path.join(GOLDEN, "st7_outputs.npz"))
    prepare(tmp_path, golden)
    run_driver(L, tmp_path, "--precision", "f32")
    want = np.array(golden["LBM_psi_60.vtk"].tobytes().decode().split("\n")[10:-1], dtype=float)
    got = np.array((tmp_path / "st_LBM_psi_60.vtk").read_text().split("\n")[10:-1], dtype=float)
    assert got.shape == want.shape
    # FP32 g after 61 steps, printed to 6 significant digits
    assert np.abs(got - want).max() <= 1e-5
