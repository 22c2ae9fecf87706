"""The lbm_cg driver against the colour-gradient program's own output files.

tests/golden/cg_outputs*.npz hold every file the reference program wrote for
variants of INPUT_cg.dat on 14x12x10 spheres with a blob phase field:
  cg_outputs.npz         reports every 50 steps to n_max = 150, density /
                         velocity VTK at 100, phase VTK every 50, mesh VTK,
                         checkpoints at 100 and at the end;
  cg_outputs_sched.npz   stabiliser, permeability window limiting the sums,
                         least-squares fit, surface-tension change, PerDir 2;
  cg_outputs_ramp.npz    a three-point body-force ramp along y, PerDir 3;
  cg_outputs_psi.npz     constant-phase faces (the initial phase) on x- and
                         x+ and y+;
  cg_outputs_cap.npz     capillary-pressure stepping of the body force along x;
  cg_outputs_restart.npz the first run's step-100 checkpoint read back and run
                         60 more steps;
  cg_outputs_pre*.npz,   pressure and velocity faces (boundary_pressure,
  cg_outputs_vel*.npz    boundary_velocity) for every Sub_BC, with the
                         stabiliser, a pressure ramp and capillary-pressure
                         stepping of the face pressures, and a restart from
                         the Sub_BC 1 run's step-100 checkpoint;
  cg_outputs_mix.npz     mixture injection on 16x12x12 spheres: the initial
                         phase of psi_mixture_ini (3-cell buffer, wetting
                         share 0.6), constant phase on x-, no surface tension
                         for x <= 4;
  cg_outputs_psi2.npz    phase faces copying the +x neighbour (flag 2) on the
                         x faces, y- and z+, the initial phase on y+;
  cg_outputs_rand*.npz   random initial phase (ini_Sat), random phase faces
                         (flag 3), and a window with a buffer phase, from the
                         program built with its clock-seeded rand() replaced
                         by the library's seeded generator (the fixture's
                         seed is passed to lbm_cg --seed);
  cg_outputs_imb.npz,    imbibition / drainage control (rel_perm_id_dir)
  cg_outputs_drain.npz   over 50 target saturations with random phase faces,
                         same seeded program.
  cg_outputs_iniv.npz    a non-zero initial velocity (inivx..z): feq(1, u0)
                         at every node, u = u0 in the first collision;
  cg_outputs_dyn.npz     input_dynamic: the INPUT file read again every 100
                         steps (input_update), its versions served in order
                         through a named pipe: force, CapA, wall colour,
                         report / output intervals, permeability, flux
                         thresholds and n_max changed during the run.
The driver, run on the same inputs at FP64, must write the same files: text
and VTK byte for byte except the wall-clock lines of Results.txt, the
checkpoints bit for bit (rows 1..).
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN

pytestmark = pytest.mark.gpu

TIMING = (b"Elapsed time is", b"The expected completion time is")
WIDTH = {"rho": 1, "velocity": 3, "f": 19, "psi": 1, "rhor": 1, "rhob": 1}


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def prepare(workdir, golden, text=None):
    from lbm_b200 import geometry as G

    shape = tuple(int(s) for s in golden["shape"])
    mask = np.unpackbits(golden["mask"])[: np.prod(shape)].reshape(shape)
    G.write_ascii(os.path.join(workdir, "mask.dat"), mask)
    (workdir / "phase.dat").write_bytes(golden["phase"].tobytes())
    (workdir / "INPUT.dat").write_text(text if text is not None else golden["input"].tobytes().decode())


def run_driver(L, workdir, *args):
    r = subprocess.run([L.driver_path("lbm_cg"), "INPUT.dat", *args], cwd=workdir, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def strip_timing(data):
    return b"\n".join(l for l in data.split(b"\n") if not l.startswith(TIMING))


def rows_digest(path, width):
    a = np.fromfile(path, dtype=np.float64).reshape(-1, width)
    return hashlib.sha256(np.ascontiguousarray(a[1:]).tobytes()).hexdigest()


def compare(tmp_path, golden, prefix):
    names = [str(n) for n in golden["names"]]
    written = sorted(n[len(prefix):] for n in os.listdir(tmp_path) if n.startswith(prefix))
    assert written == sorted(names)
    for name in names:
        path = tmp_path / (prefix + name)
        if name.startswith("LBM_checkpoint_"):
            assert rows_digest(path, WIDTH[name.split("_")[2]]) == str(golden[name]), name
        elif name == "Results.txt":
            assert strip_timing(path.read_bytes()) == strip_timing(golden[name].tobytes()), name
        else:
            assert path.read_bytes() == golden[name].tobytes(), name


FACES = ["cg_outputs_pre1.npz", "cg_outputs_pre2.npz", "cg_outputs_pre0.npz", "cg_outputs_pre3.npz",
         "cg_outputs_pre_ramp.npz", "cg_outputs_vel2.npz", "cg_outputs_vel1.npz", "cg_outputs_vel3.npz",
         "cg_outputs_cap_pre.npz"]


@pytest.mark.parametrize("fixture", ["cg_outputs.npz", "cg_outputs_sched.npz", "cg_outputs_ramp.npz",
                                     "cg_outputs_psi.npz", "cg_outputs_cap.npz", "cg_outputs_mix.npz",
                                     "cg_outputs_psi2.npz", "cg_outputs_rand.npz", "cg_outputs_rand_buf.npz",
                                     "cg_outputs_imb.npz", "cg_outputs_drain.npz", "cg_outputs_iniv.npz"] + FACES)
def test_cg_driver_writes_the_reference_files(L, fixture, tmp_path):
    golden = np.load(os.path.join(GOLDEN, fixture))
    prepare(tmp_path, golden)
    seed = ("--seed", str(int(golden["seed"]))) if "seed" in golden.files else ()
    run_driver(L, tmp_path, *seed)
    compare(tmp_path, golden, "out_")


@pytest.mark.parametrize("first_name,rst_name", [("cg_outputs.npz", "cg_outputs_restart.npz"),
                                                 ("cg_outputs_pre1.npz", "cg_outputs_pre1_restart.npz")])
def test_cg_driver_restart_matches_the_reference_restart(L, tmp_path, first_name, rst_name):
    first = np.load(os.path.join(GOLDEN, first_name))
    prepare(tmp_path, first)
    run_driver(L, tmp_path)  # writes out_LBM_checkpoint_*_100
    rst = np.load(os.path.join(GOLDEN, rst_name))
    prepare(tmp_path, rst)
    run_driver(L, tmp_path, "./out_")
    compare(tmp_path, rst, "rst_")


@pytest.mark.parametrize("fixture", ["cg_outputs.npz", "cg_outputs_pre1.npz", "cg_outputs_pre0.npz",
                                     "cg_outputs_pre2.npz", "cg_outputs_pre3.npz", "cg_outputs_vel1.npz",
                                     "cg_outputs_vel2.npz", "cg_outputs_vel3.npz", "cg_outputs_mix.npz"])
def test_cg_driver_f32_reports_match(L, tmp_path, fixture):
    golden = np.load(os.path.join(GOLDEN, fixture))
    prepare(tmp_path, golden)
    run_driver(L, tmp_path, "./", "--precision", "f32")
    want = np.loadtxt(golden["Velocity_ave_max.txt"].tobytes().decode().splitlines())
    got = np.loadtxt((tmp_path / "out_Velocity_ave_max.txt").read_text().splitlines())
    assert got.shape == want.shape
    # u_ave and u_max after up to 151 steps of FP32 populations and colour record
    assert np.allclose(got[:, :2], want[:, :2], rtol=2e-3, atol=0)
    bf_w = np.loadtxt(golden["bodyforce.txt"].tobytes().decode().splitlines())
    bf_g = np.loadtxt((tmp_path / "out_bodyforce.txt").read_text().splitlines())
    assert np.allclose(bf_g[:, :2], bf_w[:, :2], atol=3e-3)  # saturation


def test_cg_driver_reads_its_input_again(L, tmp_path):
    """input_dynamic (CG3:859-861, 5765-5925): the driver opens INPUT.dat at
    the same steps as the program and takes the same values from it."""
    from helpers import InputVersions

    golden = np.load(os.path.join(GOLDEN, "cg_outputs_dyn.npz"))
    prepare(tmp_path, golden)
    os.unlink(tmp_path / "INPUT.dat")
    keys = sorted((k for k in golden.files if k.startswith("input_version_")), key=lambda k: int(k.rsplit("_", 1)[1]))
    versions = [golden[k].tobytes().decode() for k in keys]
    with InputVersions(str(tmp_path / "INPUT.dat"), versions) as iv:
        run_driver(L, tmp_path)
        assert iv.served == len(versions)
    compare(tmp_path, golden, "out_")
