"""ctypes front-end of the oracle (TEST INFRASTRUCTURE ONLY).

Two checkers live behind this module:

* ``Restatement`` -- liboracle.so, the CPU restatement of the reference's
  single-phase sparse update (lbm_oracle.c), plus the colour-gradient and
  solute restatements.
* ``ReferenceSP3`` -- _ref/libref_sp3.so, the reference solver
  Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp compiled from
  its own source with single-rank MPI/ParMETIS stand-ins (built by the
  Makefile here when the reference sources are present; the prebuilt .so
  travels with the repository snapshot otherwise).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs may import this module.  The product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# where the fixture generators read the reference's own sample files: the
# reference project's checkout, LBM_REFERENCE_ROOT when set, else a directory
# named "reference" beside this repository's own directory
REFERENCE_ROOT = os.environ.get("LBM_REFERENCE_ROOT") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_U8P = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build(quiet=True):
    """Build liboracle.so (and _ref/ when the reference sources exist)."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _load(name):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    return C.CDLL(path)


def run_ranks(program, args, nranks, cwd, timeout=300.0):
    """Runs a reference program compiled against the multi-process MPI
    stand-in (mpishim/mpi.h) as `nranks` processes in `cwd`; returns their
    exit codes.  Messages go through a fresh directory (under /dev/shm when it
    exists); a rank still running after `timeout` seconds is killed by its pid."""
    import shutil
    import subprocess

    base = "/dev/shm" if os.path.isdir("/dev/shm") else None
    msgdir = tempfile.mkdtemp(prefix="mpishim_", dir=base)
    procs = []
    try:
        for r in range(nranks):
            env = dict(os.environ, MPISHIM_RANK=str(r), MPISHIM_SIZE=str(nranks), MPISHIM_DIR=msgdir,
                       MPISHIM_TIMEOUT=str(int(timeout)))
            log = open(os.path.join(cwd, f"rank{r}.log"), "w")
            procs.append(subprocess.Popen([program, *args], cwd=cwd, env=env, stdout=log, stderr=subprocess.STDOUT))
        codes = []
        for p in procs:
            try:
                codes.append(p.wait(timeout=timeout))
            except subprocess.TimeoutExpired:
                p.kill()
                codes.append(p.wait())
        return codes
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
        shutil.rmtree(msgdir, ignore_errors=True)


def slab_program(name):
    """Path of a slab-decomposed reference program in _ref/ (ref_sp_slab,
    ref_st7_slab), or None when it was not built."""
    path = os.path.join(HERE, "_ref", name)
    return path if os.path.exists(path) else None


def reference_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libref_sp3.so"))


class Restatement:
    """CPU restatement of the reference algorithm (lbm_oracle.c)."""

    def __init__(self):
        L = _load("liboracle.so")
        self.L = L
        L.orc_mrt_matrices.argtypes = [_F64P, _F64P]
        L.orc_mrt_matrices.restype = C.c_int
        L.orc_rates.argtypes = [C.c_double, _F64P]
        L.orc_compact.argtypes = [_U8P, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_compact.restype = C.c_int
        L.orc_nei_loc.argtypes = [_U8P, C.c_int, C.c_int, C.c_int, _I32P, C.c_int, _I32P]
        L.orc_sp_init.argtypes = [C.c_int, _F64P, _F64P, _F64P, _F64P]
        L.orc_sp_step.argtypes = [C.c_int, _I32P, _F64P, _F64P, _F64P, C.c_double, C.c_double,
                                  C.c_double, _F64P, _F64P, _F64P, _F64P, _F64P]
        L.orc_sp_error.argtypes = [C.c_int, _F64P, _F64P, C.c_int, C.c_int, C.c_int, C.c_double,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_sp_error.restype = C.c_double
        L.orc_sp_perm.argtypes = [C.c_int, _F64P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_int, _F64P,
                                  C.POINTER(C.c_double)]
        L.orc_sp_perm.restype = C.c_double
        L.orc_porosity.argtypes = [_U8P, C.c_int, C.c_int, C.c_int]
        L.orc_porosity.restype = C.c_double
        L.orc_sp_step_bc.argtypes = L.orc_sp_step.argtypes + [C.c_int, _I32P, _F64P, _I32P, _F64P, _I32P, _I32P]
        L.orc_face_list.argtypes = [_U8P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_face_list.restype = C.c_int
        L.orc_sp_perm_dp.argtypes = [C.c_int, _F64P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _F64P,
                                     C.POINTER(C.c_double)]
        L.orc_sp_perm_dp.restype = C.c_double
        L.orc_sp_dp.argtypes = [C.c_int, C.c_int, _F64P, C.c_int, C.c_int, C.c_int]
        L.orc_sp_dp.restype = C.c_double
        L.orc_sp_group_perm.argtypes = [C.c_int, _F64P, _I32P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_double, C.c_int, _I32P, _I32P, _I32P, _F64P]
        L.orc_sp_group_perm.restype = C.c_int

    def matrices(self):
        M = np.zeros((19, 19))
        MI = np.zeros((19, 19))
        ok = self.L.orc_mrt_matrices(M, MI)
        assert ok == 1
        return M, MI

    def rates(self, nu):
        S = np.zeros(19)
        self.L.orc_rates(nu, S)
        return S

    def compact(self, mask):
        nz, ny, nx = mask.shape
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        count = self.L.orc_compact(m, nx, ny, nz, None)
        coor = np.zeros(count + 1, dtype=np.int32)
        self.L.orc_compact(m, nx, ny, nz, coor.ctypes.data)
        return coor

    def nei_loc(self, mask, coor):
        nz, ny, nx = mask.shape
        count = coor.size - 1
        nei = np.zeros((count + 1) * 19, dtype=np.int32)
        self.L.orc_nei_loc(np.ascontiguousarray(mask, dtype=np.uint8), nx, ny, nz, coor, count, nei)
        return nei.reshape(count + 1, 19)

    def porosity(self, mask):
        nz, ny, nx = mask.shape
        return self.L.orc_porosity(np.ascontiguousarray(mask, dtype=np.uint8), nx, ny, nz)

    def face_list(self, mask, face):
        """Boundary-node ids of face 0..5 = x=0, x=nx-1, y=0, y=ny-1, z=0, z=nz-1."""
        nz, ny, nx = mask.shape
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        n = self.L.orc_face_list(m, nx, ny, nz, face, None)
        out = np.zeros(max(n, 1), dtype=np.int32)
        self.L.orc_face_list(m, nx, ny, nz, face, out.ctypes.data)
        return out[:n]


class Boundaries:
    """Pressure/velocity boundary settings of INPUT.dat (SP3:299-305, 318).
    Faces in INPUT order xp, xn, yp, yn, zp, zn; pre/vel 1 = on."""

    def __init__(self, sub_bc=0, in_bc=0, pre=(0,) * 6, p=(1.0,) * 6, vel=(0,) * 6, v=(0.0,) * 6):
        self.sub_bc = int(sub_bc)
        self.in_bc = int(in_bc)
        self.pre = np.array(pre, dtype=np.int32)
        self.p = np.array(p, dtype=np.float64)
        self.vel = np.array(vel, dtype=np.int32)
        self.v = np.array(v, dtype=np.float64)


class SinglePhaseRun:
    """A single-phase solve driven step by step through the restatement."""

    def __init__(self, mask, nu, g=(1e-6, 0.0, 0.0), u_init=(0.0, 0.0, 0.0), bc=None):
        self.R = Restatement()
        self.bc = bc
        self.mask = np.ascontiguousarray(mask, dtype=np.uint8)
        self.nz, self.ny, self.nx = mask.shape
        self.coor = self.R.compact(self.mask)
        self.count = self.coor.size - 1
        self.nei = np.ascontiguousarray(self.R.nei_loc(self.mask, self.coor).reshape(-1))
        self.M, self.MI = self.R.matrices()
        self.M = np.ascontiguousarray(self.M.reshape(-1))
        self.MI = np.ascontiguousarray(self.MI.reshape(-1))
        self.S = self.R.rates(nu)
        self.nu = nu
        self.g = tuple(float(x) for x in g)
        self.porosity = self.R.porosity(self.mask)
        n = self.count + 1
        self.rho = np.zeros(n)
        self.u = np.zeros(n * 3)
        self.u0 = np.zeros(n * 3)
        self.f = np.zeros(n * 19)
        self.F = np.zeros(n * 19)
        self.perm_prev = np.zeros(3)
        self.R.L.orc_sp_init(self.count, np.array(u_init, dtype=np.float64), self.rho, self.u, self.f)
        if bc is not None:
            lists = [self.R.face_list(self.mask, fc) for fc in range(6)]
            self.face_len = np.array([x.size for x in lists], dtype=np.int32)
            self.face_ids = np.ascontiguousarray(np.concatenate(lists + [np.zeros(1, np.int32)]).astype(np.int32))

    def step(self, n=1):
        for _ in range(n):
            if self.bc is None:
                self.R.L.orc_sp_step(self.count, self.nei, self.M, self.MI, self.S, *self.g,
                                     self.rho, self.u, self.u0, self.f, self.F)
            else:
                b = self.bc
                self.R.L.orc_sp_step_bc(self.count, self.nei, self.M, self.MI, self.S, *self.g,
                                        self.rho, self.u, self.u0, self.f, self.F, b.sub_bc, b.pre, b.p, b.vel,
                                        b.v, self.face_ids, self.face_len)

    def error(self):
        um = C.c_double()
        ua = C.c_double()
        e = self.R.L.orc_sp_error(self.count, self.u, self.u0, self.nx, self.ny, self.nz,
                                  self.porosity, C.byref(um), C.byref(ua))
        return e, um.value, ua.value

    def perm(self, perdir=1):
        ua = C.c_double()
        dp = 0.0
        if self.bc is not None:
            dp = self.R.L.orc_sp_dp(self.bc.in_bc, perdir, self.bc.p, self.nx, self.ny, self.nz)
        e = self.R.L.orc_sp_perm_dp(self.count, self.u, self.nx, self.ny, self.nz, self.porosity, self.nu,
                                    *self.g, dp, perdir, self.perm_prev, C.byref(ua))
        return e, self.perm_prev.copy(), ua.value

    def fields(self):
        return (self.f.reshape(-1, 19).copy(), self.u.reshape(-1, 3).copy(), self.rho.copy())

    def group_perm(self, n_sub, size, corner, dp=0.0):
        """Comput_Grop_Perm (SP:4886-5091): per cube (perm_x, perm_y, perm_z, porosity)."""
        n_sub = np.ascontiguousarray(n_sub, dtype=np.int32)
        size = np.ascontiguousarray(size, dtype=np.int32)
        corner = np.ascontiguousarray(np.asarray(corner, dtype=np.int32).reshape(-1))
        ncube = int((n_sub.astype(np.int64) ** 3).sum())
        out = np.zeros(max(ncube, 1) * 4)
        self.R.L.orc_sp_group_perm(self.count, self.u, self.coor, self.nx, self.ny, self.nz, self.nu, *self.g, dp,
                                   n_sub.size, n_sub, size, corner, out)
        return out[: ncube * 4].reshape(-1, 4)


class CGParams(C.Structure):
    _fields_ = [("nu_l", C.c_double), ("nu_g", C.c_double), ("psi_solid", C.c_double), ("cap_a", C.c_double),
                ("g", C.c_double * 3), ("body_force_phase", C.c_int), ("flux_psi", C.c_double),
                ("flux_umax", C.c_double)]


class ColourGradientRun:
    """The colour-gradient restatement (lbm_oracle_cg.c), one periodic solve."""

    def __init__(self, mask, psi, nu_l, nu_g, psi_solid, cap_a, g, body_force_phase=-1, flux_psi=0.99,
                 flux_umax=0.01):
        L = _load("liboracle.so")
        self.L = L
        L.orc_cg_matrices.argtypes = [_F64P, _F64P]
        L.orc_cg_matrices.restype = C.c_int
        L.orc_cg_nei_loc.argtypes = [_U8P, C.c_int, C.c_int, C.c_int, _I32P, C.c_int, _I32P]
        L.orc_cg_init.argtypes = [C.c_int, _F64P, np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS"),
                                  _F64P, _F64P, _F64P, _F64P, _F64P, _F64P]
        L.orc_cg_step.argtypes = [C.c_int, _I32P, _F64P, _F64P, C.POINTER(CGParams)] + [_F64P] * 10
        L.orc_cg_perm.argtypes = [C.c_int, _F64P, _F64P, C.c_int, C.c_int, C.c_int, C.c_double,
                                  C.POINTER(CGParams), _F64P, _F64P, C.POINTER(C.c_double)]
        L.orc_cg_perm.restype = C.c_double
        L.orc_cg_saturation.argtypes = [C.c_int, _F64P, C.c_int, C.c_int, C.c_int, C.c_double]
        L.orc_cg_saturation.restype = C.c_double
        R = Restatement()
        self.mask = np.ascontiguousarray(mask, dtype=np.uint8)
        self.nz, self.ny, self.nx = mask.shape
        self.coor = R.compact(self.mask)
        self.count = n = self.coor.size - 1
        self.porosity = R.porosity(self.mask)
        self.nei = np.zeros((n + 1) * 19, dtype=np.int32)
        L.orc_cg_nei_loc(self.mask, self.nx, self.ny, self.nz, self.coor, n, self.nei)
        self.M, self.MI = np.zeros(361), np.zeros(361)
        assert L.orc_cg_matrices(self.M, self.MI) == 1
        self.p = CGParams(nu_l, nu_g, psi_solid, cap_a, (C.c_double * 3)(*g), body_force_phase, flux_psi, flux_umax)
        # phase values per node in compaction order (x fastest over pore cells), as float
        flat = np.ascontiguousarray(psi, dtype=np.float64).reshape(-1)
        psi_nodes = np.zeros(n + 1, dtype=np.float32)
        psi_nodes[1:] = flat[self.mask.reshape(-1) == 0].astype(np.float32)
        z = lambda k: np.zeros(k)
        self.rho, self.psi, self.rho_r, self.rho_b = z(n + 1), z(n + 1), z(n + 1), z(n + 1)
        self.rhor, self.rhob = z(n + 1), z(n + 1)
        self.u, self.u0 = z((n + 1) * 3), z((n + 1) * 3)
        self.f, self.F = z((n + 1) * 19), z((n + 1) * 19)
        self.per_l, self.per_g = z(3), z(3)
        L.orc_cg_init(n, self.MI, psi_nodes, self.rho, self.u, self.f, self.psi, self.rho_r, self.rho_b)

    def step(self, k=1):
        for _ in range(k):
            self.L.orc_cg_step(self.count, self.nei, self.M, self.MI, C.byref(self.p), self.rho, self.u, self.u0,
                               self.f, self.F, self.psi, self.rho_r, self.rho_b, self.rhor, self.rhob)

    def perm(self):
        ua = C.c_double()
        e = self.L.orc_cg_perm(self.count, self.u, self.psi, self.nx, self.ny, self.nz, self.porosity,
                               C.byref(self.p), self.per_l, self.per_g, C.byref(ua))
        return e, self.per_l.copy(), self.per_g.copy(), ua.value

    def saturation(self):
        return self.L.orc_cg_saturation(self.count, self.psi, self.nx, self.ny, self.nz, self.porosity)

    def fields(self):
        return {"f": self.f.reshape(-1, 19).copy(), "u": self.u.reshape(-1, 3).copy(), "rho": self.rho.copy(),
                "psi": self.psi.copy(), "rho_r": self.rho_r.copy(), "rho_b": self.rho_b.copy()}


class SoluteRun:
    """D3Q7 solute restatement (lbm_oracle_st.c), periodic, fixed velocity."""

    def __init__(self, mask, c0_cells, diffusivity, u_nodes):
        L = _load("liboracle.so")
        self.L = L
        L.orc_st7_tau.argtypes = [C.c_double]
        L.orc_st7_tau.restype = C.c_double
        L.orc_st7_init.argtypes = [C.c_int, _F64P, _F64P, _F64P]
        L.orc_st7_step.argtypes = [C.c_int, _I32P, _F64P, C.c_double, _F64P, _F64P, _F64P]
        R = Restatement()
        self.mask = np.ascontiguousarray(mask, dtype=np.uint8)
        self.coor = R.compact(self.mask)
        self.count = n = self.coor.size - 1
        self.nei = np.ascontiguousarray(R.nei_loc(self.mask, self.coor).reshape(-1))
        self.tau = L.orc_st7_tau(diffusivity)
        self.u = np.ascontiguousarray(u_nodes, dtype=np.float64).reshape(-1)
        c0 = np.zeros(n + 1)
        c0[1:] = np.ascontiguousarray(c0_cells, dtype=np.float64).reshape(-1)[self.mask.reshape(-1) == 0]
        self.g, self.G, self.C = np.zeros((n + 1) * 7), np.zeros((n + 1) * 7), np.zeros(n + 1)
        L.orc_st7_init(n, c0, self.g, self.C)

    def step(self, k=1):
        for _ in range(k):
            self.L.orc_st7_step(self.count, self.nei, self.u, self.tau, self.g, self.G, self.C)

    def concentration(self):
        return self.C.copy()


def write_phase_file(path, psi):
    """Phase file of the colour-gradient solver: one value per cell, ASCII,
    x fastest (read with `fin >> pore2` into a float, CG3:2144-2150)."""
    flat = np.ascontiguousarray(psi, dtype=np.float64).reshape(-1)
    with open(path, "w") as fh:
        fh.write("\n".join(repr(float(v)) for v in flat))
        fh.write("\n")


class ReferenceCG3:
    """The reference colour-gradient solver (compiled from its source), one rank."""

    def __init__(self):
        name = os.path.join(HERE, "_ref", "libref_cg3.so")
        if not os.path.exists(name):
            build()
        if not os.path.exists(name):
            raise FileNotFoundError("libref_cg3.so not built (reference sources absent and no prebuilt library)")
        L = C.CDLL(name)
        self.L = L
        L.ref_cg3_create.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_int, C.c_double, C.c_double]
        L.ref_cg3_create.restype = C.c_int
        L.ref_cg3_step.argtypes = [C.c_int]
        L.ref_cg3_perm.argtypes = [_F64P, _F64P, C.POINTER(C.c_double)]
        L.ref_cg3_perm.restype = C.c_double
        L.ref_cg3_saturation.restype = C.c_double
        L.ref_cg3_porosity.restype = C.c_double
        L.ref_cg3_get_coor.argtypes = [_I32P]
        L.ref_cg3_get_nei_loc.argtypes = [_I32P]
        L.ref_cg3_get_f.argtypes = [_F64P]
        L.ref_cg3_get_u.argtypes = [_F64P]
        L.ref_cg3_get_scalars.argtypes = [_F64P, _F64P, _F64P, _F64P]
        L.ref_cg3_get_M.argtypes = [_F64P]
        L.ref_cg3_get_MI.argtypes = [_F64P]
        L.ref_cg3_set_mixture.argtypes = [C.c_int, C.c_double]
        self.count = 0

    def set_mixture(self, thickness, portion):
        """Mixture injection for the next create(): the reference builds the
        initial phase itself (psi_mixture_ini) instead of reading the file."""
        self.L.ref_cg3_set_mixture(int(thickness), float(portion))

    def create(self, mask, psi, nu_l, nu_g, psi_solid, cap_a, g, body_force_phase=-1, flux_psi=0.99,
               flux_umax=0.01, workdir=None):
        nz, ny, nx = mask.shape
        d = workdir or tempfile.mkdtemp(prefix="refcg3_")
        mpath = os.path.join(d, "mask.bin")
        np.ascontiguousarray(np.transpose(mask, (2, 1, 0)).astype(np.int32)).tofile(mpath)
        ppath = os.path.join(d, "phase.dat")
        write_phase_file(ppath, psi)
        self.count = self.L.ref_cg3_create(mpath.encode(), ppath.encode(), nx, ny, nz, 1, nu_l, nu_g, psi_solid,
                                           cap_a, *[float(x) for x in g], int(body_force_phase), flux_psi, flux_umax)
        return self.count

    def step(self, n=1):
        self.L.ref_cg3_step(int(n))

    def perm(self):
        pl, pg, ua = np.zeros(3), np.zeros(3), C.c_double()
        e = self.L.ref_cg3_perm(pl, pg, C.byref(ua))
        return e, pl, pg, ua.value

    def saturation(self):
        return self.L.ref_cg3_saturation()

    def coor(self):
        out = np.zeros(self.count + 1, dtype=np.int32)
        self.L.ref_cg3_get_coor(out)
        return out

    def nei_loc(self):
        out = np.zeros((self.count + 1) * 19, dtype=np.int32)
        self.L.ref_cg3_get_nei_loc(out)
        return out.reshape(-1, 19)

    def fields(self):
        n = self.count + 1
        f, u = np.zeros(n * 19), np.zeros(n * 3)
        rho, psi, rr, rb = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        self.L.ref_cg3_get_f(f)
        self.L.ref_cg3_get_u(u)
        self.L.ref_cg3_get_scalars(rho, psi, rr, rb)
        return {"f": f.reshape(-1, 19), "u": u.reshape(-1, 3), "rho": rho, "psi": psi, "rho_r": rr, "rho_b": rb}

    def matrices(self):
        M, MI = np.zeros(361), np.zeros(361)
        self.L.ref_cg3_get_M(M)
        self.L.ref_cg3_get_MI(MI)
        return M.reshape(19, 19), MI.reshape(19, 19)


class ReferenceSP3:
    """The reference solver itself (compiled from its source), one rank.

    The reference keeps its state in globals, so one instance per process is
    meaningful at a time; ``create`` re-initialises it."""

    _lib = None

    def __init__(self, fast=False):
        name = os.path.join("_ref", "libref_sp3_fast.so" if fast else "libref_sp3.so")
        if not os.path.exists(os.path.join(HERE, name)):
            build()
        if not os.path.exists(os.path.join(HERE, name)):
            raise FileNotFoundError(f"{name} not built (reference sources absent and no prebuilt library)")
        L = C.CDLL(os.path.join(HERE, name))
        self.L = L
        L.ref_sp3_create.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_double, C.c_double, C.c_double]
        L.ref_sp3_create.restype = C.c_int
        L.ref_sp3_step.argtypes = [C.c_int]
        L.ref_sp3_error.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ref_sp3_error.restype = C.c_double
        L.ref_sp3_perm.argtypes = [_F64P, C.POINTER(C.c_double)]
        L.ref_sp3_perm.restype = C.c_double
        L.ref_sp3_porosity.restype = C.c_double
        L.ref_sp3_s_v.restype = C.c_double
        for nm in ("get_f", "get_u", "get_rho", "get_M", "get_MI", "set_f", "set_u", "set_rho"):
            getattr(L, "ref_sp3_" + nm).argtypes = [_F64P]
        L.ref_sp3_get_coor.argtypes = [_I32P]
        L.ref_sp3_get_nei_loc.argtypes = [_I32P]
        L.ref_sp3_set_boundaries.argtypes = [C.c_int, C.c_int, _I32P, _F64P, _I32P, _F64P, C.c_int]
        L.ref_sp3_get_face_list.argtypes = [C.c_int, C.c_void_p]
        L.ref_sp3_get_face_list.restype = C.c_int
        self.count = 0
        self.set_boundaries(None)

    def set_boundaries(self, bc, perdir=1):
        """Boundary settings (a Boundaries, or None for the periodic path) and
        PerDir for the next create()."""
        b = bc if bc is not None else Boundaries()
        self.L.ref_sp3_set_boundaries(b.sub_bc, b.in_bc, b.pre, b.p, b.vel, b.v, int(perdir))

    def face_list(self, face):
        n = self.L.ref_sp3_get_face_list(face, None)
        out = np.zeros(max(n, 1), dtype=np.int32)
        self.L.ref_sp3_get_face_list(face, out.ctypes.data)
        return out[:n]

    def create(self, mask, nu, g=(1e-6, 0.0, 0.0), binary=True, workdir=None):
        from_path = None
        nz, ny, nx = mask.shape
        self.shape = (nx, ny, nz)
        tmpdir = workdir or tempfile.mkdtemp(prefix="refsp3_")
        from_path = os.path.join(tmpdir, "mask.bin" if binary else "mask.dat")
        if binary:
            arr = np.ascontiguousarray(np.transpose(mask, (2, 1, 0)).astype(np.int32))
            arr.tofile(from_path)
        else:
            flat = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
            out = np.empty(flat.size * 2, dtype=np.uint8)
            out[0::2] = flat + ord("0")
            out[1::2] = ord("\n")
            open(from_path, "wb").write(out.tobytes())
        self.count = self.L.ref_sp3_create(from_path.encode(), nx, ny, nz, 1 if binary else 0, nu,
                                           *[float(x) for x in g])
        return self.count

    def step(self, n=1):
        self.L.ref_sp3_step(int(n))

    def error(self):
        um = C.c_double()
        ua = C.c_double()
        e = self.L.ref_sp3_error(C.byref(um), C.byref(ua))
        return e, um.value, ua.value

    def perm(self):
        p = np.zeros(3)
        ua = C.c_double()
        e = self.L.ref_sp3_perm(p, C.byref(ua))
        return e, p, ua.value

    def coor(self):
        out = np.zeros(self.count + 1, dtype=np.int32)
        self.L.ref_sp3_get_coor(out)
        return out

    def nei_loc(self):
        out = np.zeros((self.count + 1) * 19, dtype=np.int32)
        self.L.ref_sp3_get_nei_loc(out)
        return out.reshape(-1, 19)

    def fields(self):
        n = self.count + 1
        f = np.zeros(n * 19)
        u = np.zeros(n * 3)
        r = np.zeros(n)
        self.L.ref_sp3_get_f(f)
        self.L.ref_sp3_get_u(u)
        self.L.ref_sp3_get_rho(r)
        return f.reshape(-1, 19), u.reshape(-1, 3), r

    def matrices(self):
        M = np.zeros(361)
        MI = np.zeros(361)
        self.L.ref_sp3_get_M(M)
        self.L.ref_sp3_get_MI(MI)
        return M.reshape(19, 19), MI.reshape(19, 19)

    def porosity(self):
        return self.L.ref_sp3_porosity()
