"""Pins of the boundary-condition restatement (orc_sp_step_bc, lbm_oracle.c)
against the reference's boundary_pressure / boundary_velocity.

tests/golden/sp_bc.npz was written by the reference compiled from its source
(make_golden.py --bc): 16 cases (Sub_BC 0..3 x pressure on x, pressure on
every face with a body force, velocity on every face, pressure on y with
velocity on x+ and z-), 21 steps each on 14x8x10 spheres.  The restatement
must reproduce the face lists, f, u, rho (bit for bit, by SHA-256) and the
permeability with the pressure-gradient term.  Pressure Sub_BC 3 on x alone
diverges to NaN in the reference as in the restatement (its non-equilibrium
part comes from the -y neighbour whatever the face); that case pins the NaN
path as well.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

from helpers import GOLDEN, unpack_mask

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def fixture():
    z = np.load(os.path.join(GOLDEN, "sp_bc.npz"))
    return z, unpack_mask(z["mask"], z["shape"])


def test_face_lists(oracle_mod, fixture):
    z, mask = fixture
    R = oracle_mod.Restatement()
    for fc in range(6):
        assert np.array_equal(R.face_list(mask, fc), z[f"face_{fc}"]), fc


def test_boundaries_bit_exact(oracle_mod, fixture):
    import make_golden

    z, mask = fixture
    steps = int(z["steps"])
    for name, bc, g, perdir in make_golden.bc_cases():
        run = oracle_mod.SinglePhaseRun(mask, float(z["nu"]), g, bc=bc)
        run.step(steps)
        f, u, rho = run.fields()
        want = [str(s) for s in z[name]]
        assert [digest(f[1:]), digest(u[1:]), digest(rho[1:])] == want, name
        _, perm, ua = run.perm(perdir)
        assert np.array_equal(np.array([*perm, ua]), z[name + ":perm"], equal_nan=True), name
