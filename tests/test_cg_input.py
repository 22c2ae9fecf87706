"""The colour-gradient program's INPUT file, phase file and the options the
drop-in driver refuses, on the CPU (no device calls: the checks run before
the solver is created)."""
import os

import numpy as np
import pytest

from helpers import GOLDEN


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def set_lines(text, **kv):
    lines = text.splitlines()
    for k, v in kv.items():
        i = int(k[1:])
        lines[i] = f"{v}\t\t:{lines[i].split(':', 1)[1]}"
    return "\n".join(lines) + "\n"


def test_cg_input_field_order(L):
    d = L.read_cg_input(os.path.join(GOLDEN, "INPUT_cg.dat"))
    assert (d["geometry_file"], d["phase_file"]) == ("mask.dat", "phase.dat")
    assert (d["nx"], d["ny"], d["nz"], d["n_max"], d["reso"]) == (14, 12, 10, 150, 7.0)
    assert (d["in_bc"], d["in_psi_bc"], d["gx"], d["gy"], d["gz"]) == (0, 0, 1e-5, 0.0, 0.0)
    assert (d["nu_l"], d["nu_g"], d["contact_angle"], d["cap_a"], d["permeability"]) == (0.1, 0.1, 0.70711, 1e-3,
                                                                                        2500.0)
    assert (d["wr_per"], d["perdir"], d["fre_re"], d["out_mode"], d["fre_ve"], d["fre_de"], d["fre_psi"]) == (
        1, 1, 50, 1, 100, 100, 50)
    assert d["output_path"] == "./out_"
    assert (d["stab"], d["stab_time"], d["ini_sat"], d["ini_buf"]) == (0, 500, -1.0, 0)
    assert (d["rel_perm_psi"], d["rel_perm_psi2"]) == (0.99, 0.01)
    assert (d["per_xp"], d["per_xn"], d["per_yp"], d["per_yn"], d["per_zp"], d["per_zn"]) == (10, 3, 11, 0, 9, 0)
    assert (d["fre_backup"], d["mode_backup_ini"], d["decbin"]) == (-1, 0, 0)
    assert (d["pressure_change"], d["pre_chan_pb"], d["pre_chan"]) == (0, 2, [-1] * 5)
    assert d["bodyforce_apply"] == -1
    assert (d["pressure_change2"], d["pre_chan_pb2"], d["interval_pre"], d["chan_no"], d["sat_cri"]) == (0, 1, 2000, 6,
                                                                                                        10)
    assert (d["least_square"], d["num_least_square"], d["rel_perm_id_dir"], d["rel_perm_chan_num"]) == (0, 4, 0, 5)
    assert (d["rel_perm_ift"], d["vary_ift"], d["input_dynamic"], d["update_fre"]) == (0, 0.7e-2, 0, 1000)
    assert (d["mix_psi_thickness"], d["protion_w"], d["zero_sigma_thickness"]) == (0, 0.5, 6)


def test_cg_fixture_inputs_parse(L, tmp_path):
    for name in ("cg_outputs.npz", "cg_outputs_sched.npz", "cg_outputs_ramp.npz", "cg_outputs_restart.npz"):
        g = np.load(os.path.join(GOLDEN, name))
        p = tmp_path / "INPUT.dat"
        p.write_bytes(g["input"].tobytes())
        d = L.read_cg_input(str(p))
        assert (d["nx"], d["ny"], d["nz"]) == tuple(int(s) for s in g["shape"][::-1])
        assert "Results.txt" in [str(n) for n in g["names"]]
    d = L.read_cg_input(str(p))
    assert (d["mode_backup_ini"], d["output_path"]) == (100, "./rst_")


def test_phase_file_reads_as_float(L, tmp_path):
    vals = np.array([1, -1, 0.3, 0.1234567891234, -2.5e-3, 0], dtype=np.float64)
    p = tmp_path / "phase.dat"
    p.write_text(" ".join(repr(float(v)) for v in vals[:3]) + "\n" + "\t".join(repr(float(v)) for v in vals[3:]) + "\n")
    got = L.read_phase(str(p), (3, 2, 1))
    assert got.shape == (1, 2, 3)
    assert np.array_equal(got.reshape(-1), vals.astype(np.float32).astype(np.float64))
    with pytest.raises(L.LbmError):
        L.read_phase(str(p), (7, 1, 1))


@pytest.mark.parametrize("lines,field", [
    (dict(L9="2 1.0 0 1.0"), "pre_"),
    (dict(L13="0 0.0 2 0.0"), "vel_"),
    (dict(L7=1, L15="4 0"), "psi_xp"),
    (dict(L7=1, L17="0 -1"), "psi_xp"),
    (dict(L68=20), "mix_psi_thickness"),
    (dict(L33="1 1.0 2.0"), "lattice_v"),
    (dict(L64="3 5"), "rel_perm_id_dir"),
    (dict(L64="1 0"), "rel_perm_id_dir"),
    (dict(L58="4 1 2000"), "pressure_change2"),
    (dict(L58="1 2 0"), "pressure_change2"),
    (dict(L66="1 0"), "input_dynamic"),
    (dict(L31=0), "frePsi"),
])
def test_cg_driver_refuses_options_outside_its_scope(L, tmp_path, lines, field):
    text = set_lines(open(os.path.join(GOLDEN, "INPUT_cg.dat")).read(), **lines)
    (tmp_path / "INPUT.dat").write_text(text)
    with pytest.raises(L.LbmError) as e:
        L.ColourGradient.from_input(str(tmp_path / "INPUT.dat"))
    assert e.value.status == -1 and field in str(e.value), str(e.value)


def test_st7_input_field_order_and_slab_partition(L, tmp_path):
    """The solute program's INPUT file (ST7:219-280) and its x-slab split
    (ST7:951-975) against the rank sizes the reference itself produced."""
    g = np.load(os.path.join(GOLDEN, "st7_outputs.npz"))
    p = tmp_path / "INPUT_st.dat"
    p.write_bytes(g["input"].tobytes())
    d = L.read_st7_input(str(p))
    assert (d["geometry_file"], d["conc_file"], d["nx"], d["ny"], d["nz"], d["n_max"]) == (
        "mask.dat", "phase.dat", 16, 10, 8, 60)
    assert (d["buoyancy"], d["ref_psi"], d["nu"], d["nu_s"]) == (0.0, 0.5, 0.05, 0.005)
    assert (d["fre_re"], d["out_mode"], d["fre_ve"], d["fre_psi"], d["sub_dis"], d["fre_dis"]) == (20, 1, 40, 20, 0,
                                                                                                 1000)
    assert (d["output_path"], d["fre_backup"], d["mode_backup_ini"], d["sol_ini_n"], d["decbin"]) == (
        "./st_", 40, 0, 100, 0)
    shape = tuple(int(s) for s in g["shape"])
    mask = np.unpackbits(g["mask"])[: np.prod(shape)].reshape(shape)
    first = L.slab_partition(mask, 2)
    sizes = [(mask[:, :, first[r]:first[r + 1]] == 0).sum() for r in range(2)]
    # the slab program wrote Count*3 velocities per rank
    assert sizes == [g["file:Velocity_for_solute_100.%d.bin" % r].size // 24 for r in range(2)]
    st = np.load(os.path.join(GOLDEN, "st7_slab.npz"))
    assert sizes == [int(v) for v in st["rank_nodes"]]


def test_input_versions_serve_one_text_per_opening(tmp_path):
    """The named pipe behind the input_dynamic test: each opening of the file
    by another process reads the next version whole, the last one repeats."""
    import subprocess
    import sys

    from helpers import InputVersions

    path = str(tmp_path / "INPUT.dat")
    reader = ("import sys, time\n"
              "for k in range(4):\n"
              "    print(open(sys.argv[1]).read().splitlines()[0], flush=True)\n"
              "    time.sleep(0.01)\n")
    with InputVersions(path, ["a\nx\n", "b\ny\n", "c\nz\n"]) as iv:
        r = subprocess.run([sys.executable, "-c", reader, path], capture_output=True, text=True, timeout=60)
        assert iv.served == 4
    assert r.stdout.split() == ["a", "b", "c", "c"]
    assert not os.path.exists(path)


def test_cg_dynamic_fixture_versions_parse(L, tmp_path):
    """The versions of cg_outputs_dyn.npz carry the values input_update reads
    (CG3:5780-5820): n_max, force, wall colour, CapA, permeability, the
    report / output intervals and the flux thresholds."""
    g = np.load(os.path.join(GOLDEN, "cg_outputs_dyn.npz"))
    got = []
    for k in range(5):
        p = tmp_path / f"v{k}.dat"
        p.write_bytes(g[f"input_version_{k}"].tobytes())
        d = L.read_cg_input(str(p))
        got.append((d["n_max"], d["gx"], d["contact_angle"], d["cap_a"], d["permeability"], d["fre_re"],
                    d["fre_ve"], d["fre_psi"], d["rel_perm_psi"], d["rel_perm_psi2"], d["input_dynamic"],
                    d["update_fre"]))
    assert got[0] == got[1] == (400, 1e-5, 0.70711, 1e-3, 2500.0, 50, -1, 100, 0.99, 0.01, 1, 100)
    assert got[2] == (400, 2e-5, 0.5, 2e-3, 2500.0, 50, -1, 100, 0.99, 0.01, 1, 100)
    assert got[3] == (400, 2e-5, 0.5, 2e-3, 1500.0, 25, -1, 50, 0.9, 0.02, 1, 100)
    assert got[4] == (350, 2e-5, 0.5, 2e-3, 1500.0, 25, 50, 50, 0.9, 0.02, 1, 100)
