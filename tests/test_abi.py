"""The C-ABI boundary without a GPU: the library loads, exports every entry
point include/lbm.h declares, and its host-only entry points (INPUT.dat and
geometry readers, argument checking) behave like the reference's readers."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def L():
    import __graft_entry__

    __graft_entry__.build_library()
    import lbm_b200

    return lbm_b200


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"LBM_API\s+[\w\s\*]+?\b(lbm\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol(L):
    import ctypes

    lib = L.lib()
    declared = declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    # the Python binding covers the whole ABI
    assert declared <= set(L.exported_symbols()) | {"lbm_autotune"}
    # nothing but the ABI is exported
    out = os.popen(f"nm -D --defined-only {L.LIB_PATH}").read()
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert exported == declared
    assert lib.lbm_abi_version() == 1
    assert lib.lbm_status_string(-6).decode() == "not converged"
    del ctypes


def test_read_input_field_order(L):
    d = L.read_input(os.path.join(GOLDEN, "INPUT_sp.dat"))
    assert d["geometry_file"] == "mask_24.dat"
    assert (d["nx"], d["ny"], d["nz"]) == (24, 20, 16)
    assert d["n_max"] == 4999 and d["reso"] == 7.5 and d["in_bc"] == 0
    assert (d["gx"], d["gy"], d["gz"]) == (2.5e-6, -1.0e-7, 3.0e-7)
    assert (d["pre_yp"], d["p_yp"], d["pre_yn"], d["p_yn"]) == (0, 1.1, 0, 1.2)
    assert (d["v_xp"], d["v_zn"]) == (0.01, 0.09)
    assert d["in_vis"] == 0.16666666666666667
    assert (d["inivx"], d["inivy"], d["inivz"]) == (1.0e-5, 2.0e-5, -3.0e-5)
    assert (d["wr_per"], d["perdir"], d["fre_re"], d["out_mode"], d["fre_ve"], d["fre_de"]) == (1, 2, 100, 1, -1, 0)
    assert (d["lattice_v"], d["dx_input"], d["dt_input"]) == (0, 1.0, 2.0)
    assert d["output_path"] == "./out_"
    assert (d["sub_bc"], d["loc_perm"]) == (2, 0)
    assert (d["par_per_x"], d["par_per_y"], d["par_per_z"]) == (1, 0, 1)
    assert (d["per_xp"], d["per_xn"], d["per_yp"], d["per_yn"], d["per_zp"], d["per_zn"]) == (20, 3, 19, 0, 12, 2)
    assert (d["fre_backup"], d["mode_backup_ini"], d["vel_sol"]) == (-1, 0, -1)
    assert d["n_gperm"] == [1, 1, 2, 4] and d["size_gperm"] == [512, 256, 128, 64]
    assert d["c_gperm"] == [[0, 1, 1], [128, 129, 130], [131, 132, 133], [134, 135, 136]]
    assert d["decbin"] == 0 and d["nnf_module"] == 0 and (d["nnf_m"], d["nnf_n"]) == (0.001, 0.25)


def test_read_input_errors(L, tmp_path):
    with pytest.raises(L.LbmError) as e:
        L.read_input(str(tmp_path / "missing.dat"))
    assert e.value.status == -2
    bad = tmp_path / "bad.dat"
    bad.write_text("header\nmask.dat :file\nx y z :bad\n")
    with pytest.raises(L.LbmError) as e:
        L.read_input(str(bad))
    assert e.value.status == -7


def test_read_mask_formats(L, tmp_path):
    from lbm_b200 import geometry as G

    mask = G.overlapping_spheres((13, 7, 5), 0.5, 2.0, seed=3)
    G.write_ascii(tmp_path / "m.dat", mask)
    G.write_binary(tmp_path / "m.bin", mask)
    a = L.read_mask(str(tmp_path / "m.dat"), (13, 7, 5), 0)
    b = L.read_mask(str(tmp_path / "m.bin"), (13, 7, 5), 1)
    assert np.array_equal(a, mask) and np.array_equal(b, mask)
    assert np.array_equal(G.read_ascii(tmp_path / "m.dat", (13, 7, 5)), mask)
    assert np.array_equal(G.read_binary(tmp_path / "m.bin", (13, 7, 5)), mask)
    # SP3 treats any non-zero token as solid (Partition_Solid: Solid == 0 is pore)
    (tmp_path / "t.dat").write_text("0 2\n-1 0\n1 0 0 0")
    t = L.read_mask(str(tmp_path / "t.dat"), (2, 2, 2), 0)
    assert t.reshape(-1).tolist() == [0, 1, 1, 0, 1, 0, 0, 0]
    with pytest.raises(L.LbmError) as e:
        L.read_mask(str(tmp_path / "t.dat"), (3, 3, 3), 0)  # too few tokens
    assert e.value.status == -7
    with pytest.raises(L.LbmError) as e:
        L.read_mask(str(tmp_path / "m.bin"), (13, 7, 6), 1)  # short binary file
    assert e.value.status == -7
    with pytest.raises(L.LbmError) as e:
        L.read_mask(str(tmp_path / "none.dat"), (2, 2, 2), 0)
    assert e.value.status == -2


def test_create_argument_checks(L):
    mask = np.zeros((4, 4, 4), dtype=np.uint8)
    with pytest.raises(L.LbmError) as e:
        L.SinglePhase(mask, nu=-1.0)
    assert e.value.status == -1
    with pytest.raises(L.LbmError) as e:
        L.SinglePhase(mask, nu=0.1, precision=9)
    assert e.value.status == -1


def test_create_without_gpu_fails_loudly(L):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(L.LbmError) as e:
        L.SinglePhase(np.zeros((4, 4, 4), dtype=np.uint8), nu=0.1)
    assert e.value.status == -10
