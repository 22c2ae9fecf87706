"""The lbm_sp driver against the reference program's own output files.

tests/golden/sp_outputs.npz holds every file the reference program wrote for
one INPUT.dat (14x12x10 spheres, n_max=250, reports every 50 steps, VTK every
100, checkpoints every 100 and at the end, solute velocity at 200);
sp_outputs_bc.npz the same for pressure faces on x (Sub_BC 2, in_BC 1);
sp_outputs_lat.npz and sp_outputs_lat2.npz the same with a self-defined
lattice velocity (dx, dt = 1, 2 and 1, 1/2: lat_c = 1/2 and 2),
sp_outputs_bc_lat.npz the pressure faces at lat_c = 1/2 and
sp_outputs_vel_lat.npz a velocity inlet with a pressure outlet (Sub_BC 1) at
lat_c = 2.  The
driver, run on the same INPUT.dat and mask at FP64, must write the same files:
text and VTK byte for byte (except the wall-clock lines of Results.txt), the
checkpoints and the solute velocity bit for bit (rows 1..; row 0 of the
reference's rho and velocity checkpoints is uninitialised memory).

Restart: a run restored from the step-200 checkpoint and advanced 60 steps
equals a continuous 261-step run bit for bit.  (The reference's own restart
divides by an unset global, SP3:3663, and stops with NaN; it is not compared.)
"""
import hashlib
import os
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


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "sp_outputs.npz"))


def set_lines(text, **kv):
    lines = text.splitlines()
    for k, v in kv.items():
        i = int(k[1:])
        lines[i] = f"{v}\t\t:{lines[i].split(':', 1)[1]}"
    return "\n".join(lines) + "\n"


def prepare(workdir, golden, text=None):
    from lbm_b200 import geometry as G

    shape = tuple(int(s) for s in golden["shape"])
    mask = np.unpackbits(golden["mask"])[: np.prod(shape)].reshape(shape)
    G.write_ascii(os.path.join(workdir, "mask.dat"), mask)
    with open(os.path.join(workdir, "INPUT.dat"), "w") as f:
        f.write(text if text is not None else golden["input"].tobytes().decode())


def run_driver(L, workdir, *args):
    r = subprocess.run([L.driver_path(), "INPUT.dat", *args], cwd=workdir, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def strip_timing(data):
    return b"\n".join(l for l in data.split(b"\n") if not l.startswith(TIMING))


def normalise(name, data):
    """Drops what the reference leaves to chance: the wall-clock lines of
    Results.txt, and the relative change on the first line of the
    permeability file, which divides by the never-set Permia (SP3:469, 3615)."""
    if name == "Results.txt":
        return strip_timing(data)
    if name == "Permeability_error_local_Perm.txt":
        lines = data.split(b"\n")
        lines[0] = lines[0].split(b" ")[0]
        return b"\n".join(lines)
    return data


def rows_digest(path, width):
    a = np.fromfile(path, dtype=np.float64).reshape(-1, width)
    return hashlib.sha256(np.ascontiguousarray(a[1:]).tobytes()).hexdigest()


@pytest.mark.parametrize("fixture", ["sp_outputs.npz", "sp_outputs_bc.npz", "sp_outputs_lat.npz",
                                     "sp_outputs_lat2.npz", "sp_outputs_bc_lat.npz", "sp_outputs_vel_lat.npz"])
def test_driver_writes_the_reference_files(L, fixture, tmp_path):
    golden = np.load(os.path.join(GOLDEN, fixture))
    prepare(tmp_path, golden)
    run_driver(L, tmp_path)
    names = [str(n) for n in golden["names"]]
    written = sorted(n[len("out_"):] for n in os.listdir(tmp_path) if n.startswith("out_"))
    assert written == sorted(names)
    for name in names:
        path = tmp_path / ("out_" + name)
        if name.startswith("LBM_checkpoint_"):
            width = {"rho": 1, "velocity": 3, "f": 19}[name.split("_")[2]]
            assert rows_digest(path, width) == str(golden[name]), name
        elif name.startswith("Velocity_for_solute_"):
            got = hashlib.sha256(np.fromfile(path, dtype=np.float64).tobytes()).hexdigest()
            assert got == str(golden[name]), name
        else:
            want = normalise(name, golden[name].tobytes())
            got = normalise(name, path.read_bytes())
            assert got == want, name


def test_restart_continues_the_trajectory(L, golden, tmp_path):
    text = golden["input"].tobytes().decode()
    prepare(tmp_path, golden)
    run_driver(L, tmp_path)  # writes out_LBM_checkpoint_*_200
    rst = set_lines(text, L3=59, L18=30, L20=-1, L21=-1, L24="./rst_", L32=0, L33=200, L34=-1)
    prepare(tmp_path, golden, rst)
    run_driver(L, tmp_path, "./out_")
    cont = set_lines(text, L3=260, L18=65, L20=-1, L21=-1, L24="./cont_", L32=0, L34=-1)
    prepare(tmp_path, golden, cont)
    run_driver(L, tmp_path)
    for what, width in (("f", 19), ("rho", 1), ("velocity", 3)):
        a = rows_digest(tmp_path / f"rst_LBM_checkpoint_{what}_59.0.bin_input", width)
        b = rows_digest(tmp_path / f"cont_LBM_checkpoint_{what}_260.0.bin_input", width)
        assert a == b, what


def test_driver_f32_reports_match(L, golden, tmp_path):
    prepare(tmp_path, golden)
    run_driver(L, tmp_path, "./", "--precision", "f32")
    want = np.loadtxt(golden["Velocity_ave_max.txt"].tobytes().decode().splitlines())
    got = np.loadtxt((tmp_path / "out_Velocity_ave_max.txt").read_text().splitlines())
    assert got.shape == want.shape
    # u_ave, u_max and the max relative change of u: FP32 storage of f - w
    assert np.allclose(got[:, :2], want[:, :2], rtol=1e-4, atol=0)
    assert np.allclose(got[:, 2], want[:, 2], rtol=1e-3, atol=0)
    perm_w = np.loadtxt(golden["Permeability_error_local_Perm.txt"].tobytes().decode().splitlines())
    perm_g = np.loadtxt((tmp_path / "out_Permeability_error_local_Perm.txt").read_text().splitlines())
    assert np.allclose(perm_g[:, 0], perm_w[:, 0], rtol=1e-4, atol=0)


@pytest.mark.parametrize("fixture", ["sp_outputs_lat.npz", "sp_outputs_lat2.npz", "sp_outputs_bc_lat.npz",
                                     "sp_outputs_vel_lat.npz"])
@pytest.mark.parametrize("precision,rtol", [("f64fast", 2e-5), ("f32", 1e-4), ("f16", 2e-3)])
def test_driver_lattice_reports_match(L, fixture, precision, rtol, tmp_path):
    """The deviation-storage kernels step a self-defined lattice in units of
    lat_c (force dt g / lat_c, velocities scaled by lat_c on the way in and
    out, face rules on the unit lattice): the six-digit reports of FP64 and
    FP32 in that form match the reference's (to the last printed digit on
    every fixture so far; 1e-4 allows a flipped rounding), FP16's to its
    storage precision (1.2e-4 - 6.1e-4 measured)."""
    golden = np.load(os.path.join(GOLDEN, fixture))
    prepare(tmp_path, golden)
    run_driver(L, tmp_path, "./", "--precision", precision)
    want = np.loadtxt(golden["Velocity_ave_max.txt"].tobytes().decode().splitlines())
    got = np.loadtxt((tmp_path / "out_Velocity_ave_max.txt").read_text().splitlines())
    assert got.shape == want.shape
    assert np.allclose(got[:, :2], want[:, :2], rtol=rtol, atol=0)
    perm_w = np.loadtxt(golden["Permeability_error_local_Perm.txt"].tobytes().decode().splitlines())
    perm_g = np.loadtxt((tmp_path / "out_Permeability_error_local_Perm.txt").read_text().splitlines())
    assert np.allclose(perm_g[:, 0], perm_w[:, 0], rtol=rtol, atol=0)


def test_set_lattice_only_before_the_first_step(L):
    from helpers import spheres

    m = spheres((16, 14, 12), 0.5, 3.0, seed=2)
    with L.SinglePhase(m, 1 / 6, (1e-5, 0.0, 0.0), precision="f64") as s:
        s.set_lattice(1.0, 2.0)
        s.step(3)
        with pytest.raises(L.LbmError):
            s.set_lattice(1.0, 1.0)
    with L.SinglePhase(m, 1 / 6, (1e-5, 0.0, 0.0), precision="f32") as s:
        with pytest.raises(L.LbmError):
            s.set_lattice(0.0, 1.0)
