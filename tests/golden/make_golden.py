"""Generates the golden fixtures of this directory by running the reference
solver itself: Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp
compiled from its own source (oracle/Makefile -> oracle/_ref/libref_sp3.so).

    python tests/golden/make_golden.py [--cfg1 | --cg | --outputs | --cg-outputs | --bc | --st7 | --st7-outputs |
                                        --slab-perm]

Fixtures (all inputs are stored with the outputs, so nothing depends on a
random generator at test time):
  sp_outputs.npz  the reference program itself (oracle/_ref/ref_sp3_main)
                run on an INPUT.dat: every file it writes  (--outputs)
  sp_outputs_bc.npz  the same with pressure faces on x (Sub_BC 2, in_BC 1)  (--outputs)
  sp_outputs_lat*.npz  the same with a self-defined lattice velocity  (--outputs)
  cg_small.npz  colour-gradient reference, see cg_small()  (--cg)
  cg_outputs*.npz  the colour-gradient program (oracle/_ref/ref_cg3_main) on
                INPUT_cg.dat variants: every file it writes, and a restart from
                its checkpoint, see cg_program_outputs()  (--cg-outputs)
  sp_bc.npz     pressure/velocity boundaries, Sub_BC 0..3, see bc_fixture()  (--bc)
  st7_slab.npz  the solute program at two ranks, see st7_fixture()  (--st7)
  st7_outputs*.npz  every file the solute program writes at two ranks (both
                output layouts, and a restart), see st7_program_outputs()
                (--st7-outputs)
  sp_slab_perm.npz  the slab single-phase program at two ranks with its
                local and group permeabilities, see slab_perm_fixture()  (--slab-perm)
  sp_small.npz  12x10x8 overlapping spheres, 20 steps: compaction, nei_loc,
                M^-1, f/u/rho after 20 steps, Error and Comput_Perm outputs
  sp_24.npz     24^3 spheres, 200 steps: compaction digest, u, rho, f digest,
                diagnostics
  sp_cfg1.npz   64^3 spheres r=6, porosity 0.40, nu=1/6 (tau=1), gx=1e-6,
                5000 steps (the reference's n_max=4999): diagnostics every 500
                steps, digests of f and u, u of every 97th node  (--cfg1; ~8 min)
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "jianhui-lbm_b200"))
sys.path.insert(0, os.path.dirname(HERE))  # tests/: helpers

import oracle  # noqa: E402
from lbm_b200 import geometry as G  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def pack(mask):
    return np.packbits(mask.reshape(-1).astype(np.uint8))


def diag(ref):
    e, umax, umean = ref.error()
    pe, perm, uave = ref.perm()
    return np.array([e, umax, umean, pe, perm[0], perm[1], perm[2], uave])


def small(ref):
    mask = G.overlapping_spheres((12, 10, 8), 0.6, 2.5, seed=11)
    nu, g, steps = 0.1, (1e-5, 2e-6, -1e-6), 20
    ref.create(mask, nu, g, binary=True)
    coor, nei = ref.coor(), ref.nei_loc()
    _, MI = ref.matrices()
    ref.step(steps)
    d = diag(ref)
    f, u, rho = ref.fields()
    np.savez_compressed(os.path.join(HERE, "sp_small.npz"), mask=pack(mask), shape=np.array(mask.shape), nu=nu,
                        g=np.array(g), steps=steps, coor=coor, nei_loc=nei, MI=MI, f=f, u=u, rho=rho, diag=d)
    print("sp_small", mask.shape, ref.count)


def mid(ref):
    mask = G.overlapping_spheres((24, 24, 24), 0.55, 4.0, seed=5)
    nu, g, steps = 0.05, (1e-5, 0.0, 0.0), 200
    ref.create(mask, nu, g, binary=False)  # exercises the ASCII reader too
    coor = ref.coor()
    nei = ref.nei_loc()
    ref.step(steps - 1)
    ref.step(1)
    d = diag(ref)
    f, u, rho = ref.fields()
    np.savez_compressed(os.path.join(HERE, "sp_24.npz"), mask=pack(mask), shape=np.array(mask.shape), nu=nu,
                        g=np.array(g), steps=steps, coor_digest=digest(coor), nei_digest=digest(nei), u=u, rho=rho,
                        f_digest=digest(f), u_digest=digest(u), f_sample=f[1::53].copy(), diag=d)
    print("sp_24", mask.shape, ref.count)


def cfg1(ref):
    mask = G.overlapping_spheres((64, 64, 64), 0.40, 6.0, seed=2024)
    nu, g, steps, every = 0.16666666666666667, (1e-6, 0.0, 0.0), 5000, 500
    ref.create(mask, nu, g, binary=True)
    hist = []
    done = 0
    while done < steps:
        ref.step(every)
        done += every
        hist.append([done] + list(diag(ref)))
        print("cfg1", done, hist[-1][1:], flush=True)
    f, u, rho = ref.fields()
    np.savez_compressed(os.path.join(HERE, "sp_cfg1.npz"), mask=pack(mask), shape=np.array(mask.shape), nu=nu,
                        g=np.array(g), steps=steps, every=every, history=np.array(hist), f_digest=digest(f),
                        u_digest=digest(u), rho_digest=digest(rho), u_sample=u[1::97].copy(),
                        f_sample=f[1::997].copy(), count=ref.count, porosity=ref.porosity())


CG_ARGS = dict(nu_l=0.1, nu_g=0.1, psi_solid=0.70711, cap_a=1e-3, g=(1e-5, 0.0, 0.0), body_force_phase=-1,
               flux_psi=0.99, flux_umax=0.01)


def cg_small():
    """Colour-gradient reference (CG3) on 18x16x14 random cylinders with a
    blob phase field (saturation 0.5), 60 steps."""
    mask = G.random_cylinders((18, 16, 14), 0.6, 2.0, seed=31)
    psi = G.blob_phase_field(mask, seed=32, saturation=0.5)
    ref = oracle.ReferenceCG3()
    ref.create(mask, psi, **CG_ARGS)
    coor, nei = ref.coor(), ref.nei_loc()
    ref.step(60)
    d = ref.fields()
    e, pl, pg, ua = ref.perm()
    sat = ref.saturation()
    np.savez_compressed(os.path.join(HERE, "cg_small.npz"), mask=pack(mask), shape=np.array(mask.shape), psi0=psi,
                        steps=60, coor=coor, nei_loc=nei, f=d["f"], u=d["u"], rho=d["rho"], psi=d["psi"],
                        rho_r=d["rho_r"], rho_b=d["rho_b"], perm_l=pl, perm_g=pg, u_ave=ua, saturation=sat,
                        args=np.array([CG_ARGS["nu_l"], CG_ARGS["nu_g"], CG_ARGS["psi_solid"], CG_ARGS["cap_a"],
                                       *CG_ARGS["g"], CG_ARGS["body_force_phase"], CG_ARGS["flux_psi"],
                                       CG_ARGS["flux_umax"]]))
    print("cg_small", mask.shape, ref.count)


def input_text(**kv):
    """INPUT.dat for the reference program: INPUT_sp.dat with some values
    replaced; keys are the 0-based line numbers of the file."""
    lines = open(os.path.join(HERE, "INPUT_sp.dat")).read().splitlines()
    for i, v in kv.items():
        lines[int(i[1:])] = f"{v}\t\t:{lines[int(i[1:])].split(':', 1)[1]}"
    return "\n".join(lines) + "\n"


# Files the reference program writes; rows 0 of the rho/velocity checkpoints
# are uninitialised memory in the reference and are not compared.
TEXT_OUTPUTS = ["Results.txt", "Permeability_error_local_Perm.txt", "Velocity_ave_max.txt", "bodyforce.txt",
                "General_Results.txt"]


def run_program(workdir, input_txt, mask, args=()):
    import subprocess

    exe = os.path.join(ROOT, "oracle", "_ref", "ref_sp3_main")
    G.write_ascii(os.path.join(workdir, "mask.dat"), mask)
    with open(os.path.join(workdir, "INPUT.dat"), "w") as f:
        f.write(input_txt)
    subprocess.run([exe, "INPUT.dat", *args], cwd=workdir, check=True, capture_output=True)


def collect(workdir, prefix="out_"):
    out = {}
    for name in sorted(os.listdir(workdir)):
        if not name.startswith(prefix):
            continue
        key = name[len(prefix):]
        data = open(os.path.join(workdir, name), "rb").read()
        if key.startswith("LBM_checkpoint_"):
            width = {"rho": 1, "velocity": 3, "f": 19}[key.split("_")[2]]
            out[key] = digest(np.frombuffer(data, dtype=np.float64).reshape(-1, width)[1:])
        elif key.startswith("Velocity_for_solute_"):
            out[key] = digest(np.frombuffer(data, dtype=np.float64))
        else:
            out[key] = data
    return out


def program_outputs(only=None):
    """The reference program run end to end on 14x12x10 spheres: 251 steps
    (n_max=250) writing every output family (reports every 50 steps, VTK
    every 100, checkpoints every 100 and at the end, solute velocity at 200).
    Stored: the INPUT file, the mask, text and VTK outputs verbatim, sha256 of
    checkpoint rows 1.. and of the solute velocity file.

    The reference's restart path (USE BACKUP DATA) is not recorded: its
    Backup_init (SP3:3663) divides by the global Zoom, which only init() sets,
    so a restarted run has dt = dx = inf and stops at its first report with
    NaN."""
    mask = G.overlapping_spheres((14, 12, 10), 0.6, 2.5, seed=21)
    base = dict(L1="mask.dat", L2="14 12 10", L3=250, L17=1, L18=50, L20=100, L21=100, L32=100, L34=200)
    runs = [("sp_outputs.npz", input_text(**base))]
    # pressure faces on x (Sub_BC 2, in_BC 1: the permeability includes the
    # pressure gradient), no body force: reports every 50 steps, velocity VTK
    # at 150
    bc = dict(L1="mask.dat", L2="14 12 10", L3=150, L4=7.5, L5=1, L6="0 0 0", L7="1 1.0 1 1.005", L17=1, L18=50,
              L20=150, L21=-1, L25=2, L32=-1, L34=-1)
    runs.append(("sp_outputs_bc.npz", input_text(**bc)))
    # self-defined lattice velocity: dx = 1, dt = 2 (lat_c = 1/2, tau = 1.5)
    # and dx = 1, dt = 1/2 (lat_c = 2, tau = 0.75), with the template's
    # initial velocity and three-component force
    runs.append(("sp_outputs_lat.npz", input_text(**base, L23="1 1.0 2.0")))
    runs.append(("sp_outputs_lat2.npz", input_text(**base, L23="1 1.0 0.5")))
    # the same lattices with faces: the pressure faces above at lat_c = 1/2,
    # and a velocity inlet on x- (0.0005) with a pressure outlet on x+
    # (Sub_BC 1; the unused p_xn = 1.002 still enters Comput_Perm's pressure
    # term, SP3:3543-3556) at lat_c = 2, dt = 1/2
    runs.append(("sp_outputs_bc_lat.npz", input_text(**bc, L23="1 1.0 2.0")))
    vel = dict(bc, L7="1 1.0 0 1.002", L10="0 0.0 1 0.0005", L25=1, L23="1 1.0 0.5")
    runs.append(("sp_outputs_vel_lat.npz", input_text(**vel)))
    for fname, text in runs:
        if only is None or only in fname:
            save_program_outputs(fname, mask, text)


def save_program_outputs(fname, mask, input_txt):
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        run_program(d, input_txt, mask)
        a = collect(d, "out_")
    blob = {"mask": pack(mask), "shape": np.array(mask.shape), "input": np.frombuffer(input_txt.encode(), np.uint8),
            "names": np.array(sorted(a))}
    for k, v in a.items():
        blob[k] = np.frombuffer(v, np.uint8) if isinstance(v, bytes) else np.array(v)
    np.savez_compressed(os.path.join(HERE, fname), **blob)
    print(fname, sorted(a))


def cg_input_text(**kv):
    """INPUT file of the colour-gradient program: INPUT_cg.dat with some
    values replaced; keys are the 0-based line numbers of the file."""
    lines = open(os.path.join(HERE, "INPUT_cg.dat")).read().splitlines()
    for i, v in kv.items():
        lines[int(i[1:])] = f"{v}\t\t:{lines[int(i[1:])].split(':', 1)[1]}"
    return "\n".join(lines) + "\n"


def cg_geometry():
    """14x12x10 spheres (porosity 0.6) with a blob phase field at S_w = 0.5."""
    mask = G.overlapping_spheres((14, 12, 10), 0.6, 2.5, seed=21)
    psi = G.blob_phase_field(mask, seed=22, saturation=0.5)
    return mask, psi


def cg_mix_geometry():
    """16x12x12 spheres (porosity 0.6) for the mixture-injection run: ny = nz,
    so the reference's ring walk of the mixture initialisation (rings up to
    max(ny, nz)/2 around the plane's centre) stays inside the plane.  The
    phase file is not read with mixture injection; it is written all +1."""
    mask = G.overlapping_spheres((16, 12, 12), 0.6, 2.5, seed=31)
    return mask, np.ones(mask.shape)


def phase_text(psi):
    return " ".join(str(int(v)) for v in psi.reshape(-1)) + "\n"


# The colour-gradient program's runs (the reference program compiled from its
# source, oracle/_ref/ref_cg3_main), name -> INPUT line overrides.
CG_RUNS = {
    # reports every 50 steps to n_max = 150, VTK of density / velocity at 100,
    # phase VTK every 50, mesh VTK, checkpoints at 100 and at the end
    "cg_outputs.npz": dict(L45=100),
    # stabiliser (force from step 30), permeability window 3..10 on x limiting
    # the sums, least-squares fit over 4 reports, surface tension changed at
    # step 100, y the permeability direction, the force on both phases, a
    # second force component; reports every 25 steps
    "cg_outputs_sched.npz": dict(L8="1.0e-5 4.0e-6 0.0", L26=2, L27=25, L28=0, L29=-1, L30=-1, L31=75, L36="1 30",
                                 L40="1 0 0", L41="10 3", L56=0, L62="1 4", L65="100 2.0e-3"),
    # body-force ramp along y through three points (the first segment starts
    # from gx, as the reference writes it), z the permeability direction
    # constant-phase faces of the initial phase on both x faces and the y+
    # face (in_psi_BC = 1, the reference's sample input turns the x faces on),
    # checkpoint at the end only
    "cg_outputs_psi.npz": dict(L7=1, L15="1 1", L16="1 0", L29=-1, L30=-1, L45=0),
    # phase faces copying the +x neighbour's phase (flag 2) on both x faces,
    # y- and z+ (their copies run along x inside the face), the initial phase
    # on y+; phase VTK every 50 steps
    "cg_outputs_psi2.npz": dict(L7=1, L15="2 2", L16="1 2", L17="2 0", L29=-1, L30=-1, L45=0),
    # capillary-pressure stepping along x with the body force: three steps
    # of 30 steps each towards 3e-5, the next one after two reports in a row
    # with the saturation changing by less than 1e-2; reports every 10 steps
    "cg_outputs_cap.npz": dict(L4=250, L27=10, L28=0, L29=-1, L30=-1, L31=-1, L58="1 2 30",
                               L59="1.0 0.993 3e-5 3 2", L60="1e-2"),
    "cg_outputs_ramp.npz": dict(L8="1.0e-5 2.0e-6 -1.0e-6", L26=3, L27=25, L28=0, L29=-1, L30=-1, L31=-1,
                                L50="2 2", L51="40 1.0 1.0 8.0e-6", L52="90 1.0 1.0 3.0e-6",
                                L53="120 1.0 1.0 5.0e-6"),
    # pressure/velocity faces (boundary_pressure / boundary_velocity), one
    # Sub_BC per run, no body force unless named:
    # Sub_BC 1 pressure on both x faces with constant-phase x faces; the
    # step-100 checkpoint also seeds a restart (cg_outputs_pre1_restart.npz)
    "cg_outputs_pre1.npz": dict(L6=1, L7=1, L8="0.0 0.0 0.0", L9="1 1.0 1 1.004", L15="1 1", L35=1, L29=-1,
                                L30=-1, L45=100),
    # Sub_BC 2 (moments of the inner neighbour) on the y faces with a body
    # force along x; stabiliser from step 30 holds force and faces back
    "cg_outputs_pre2.npz": dict(L6=1, L8="5.0e-6 0.0 0.0", L10="1 1.0 1 1.003", L26=2, L35=2, L36="1 30",
                                L29=-1, L30=-1, L31=-1),
    # Sub_BC 0 (rest equilibrium) on the z faces, z the permeability direction
    "cg_outputs_pre0.npz": dict(L6=1, L8="0.0 0.0 0.0", L11="1 1.0 1 1.002", L26=3, L35=0, L29=-1, L30=-1,
                                L31=-1),
    # Sub_BC 3 (non-equilibrium part of the -y neighbour) on the y faces
    "cg_outputs_pre3.npz": dict(L6=1, L8="0.0 0.0 0.0", L10="1 1.0 1 1.002", L26=2, L35=3, L29=-1, L30=-1,
                                L31=-1),
    # Sub_BC 1 on the x faces with a pressure ramp along x through three
    # points, reports every 25 steps
    "cg_outputs_pre_ramp.npz": dict(L6=1, L8="0.0 0.0 0.0", L9="1 1.0 1 1.004", L35=1, L27=25, L29=-1, L30=-1,
                                    L31=-1, L50="1 1", L51="40 1.0 1.006 0.0", L52="90 1.0 1.002 0.0",
                                    L53="120 1.0 1.004 0.0"),
    # Sub_BC 2 velocity (non-equilibrium bounce-back; the x flags act on the
    # z faces) with in_BC off
    "cg_outputs_vel2.npz": dict(L8="0.0 0.0 0.0", L12="1 0.002 1 0.002", L35=2, L29=-1, L30=-1, L31=-1),
    # Sub_BC 1 velocity (equilibrium) on the y faces and Sub_BC 1 pressure on
    # the x faces together
    "cg_outputs_vel1.npz": dict(L6=1, L8="0.0 0.0 0.0", L9="1 1.0 1 1.002", L13="1 0.001 1 0.001", L35=1,
                                L29=-1, L30=-1, L31=-1),
    # Sub_BC 3 velocity (density of the inner neighbour) on the x faces
    "cg_outputs_vel3.npz": dict(L8="0.0 0.0 0.0", L12="1 0.002 1 0.002", L35=3, L29=-1, L30=-1, L31=-1),
    # initial velocity (inivx..z): every node starts from feq(1, u0), the
    # first collision takes u = u0; reports every 25 steps, phase VTK every 50
    "cg_outputs_iniv.npz": dict(L22="1.0e-3 -5.0e-4 2.0e-4", L27=25, L29=-1, L30=-1, L45=0),
    # capillary-pressure stepping with the face pressures along x (Sub_BC 1)
    "cg_outputs_cap_pre.npz": dict(L4=250, L6=1, L8="0.0 0.0 0.0", L9="1 1.0 1 1.0", L35=1, L27=10, L28=0,
                                   L29=-1, L30=-1, L31=-1, L58="1 1 30", L59="1.0 1.006 2e-5 3 2", L60="1e-2"),
}


# Runs on their own geometry: name -> (geometry function, INPUT overrides).
CG_GEOMETRY_RUNS = {
    # mixture injection: initial phase from psi_mixture_ini with a 3-cell
    # buffer and a wetting share of 0.6 next to the solid, constant phase on
    # the x- face, no surface tension for x <= 4; reports every 25 steps,
    # phase VTK every 50, checkpoints at the end
    "cg_outputs_mix.npz": (cg_mix_geometry, dict(L3="16 12 12", L7=1, L15="0 1", L68=3, L69=0.6, L70=4,
                                                  L27=25, L29=-1, L30=-1, L45=0)),
}


# Runs with input_dynamic (the INPUT file read again every 100 steps,
# input_update): name -> the line overrides of each version, in the order the
# program opens the file (at start, then at steps 0, 100, 200, 300).  Base:
# 400 steps, reports every 50, phase VTK every 100, the stabiliser holding the
# force back to step 150 (the update at step 0 turns it on, gxs = gx),
# checkpoints at the end.  Step 100: force doubled, CapA 2e-3, wall colour
# 0.5.  Step 200: reports every 25, single-phase permeability 1500 mD, flux
# thresholds 0.9 / 0.02, phase VTK every 50.  Step 300: n_max 350, velocity
# VTK every 50.
CG_DYNAMIC_BASE = dict(L4=400, L27=50, L29=-1, L30=-1, L31=100, L36="1 150", L45=0, L66="1 100")
CG_DYNAMIC_RUNS = {
    "cg_outputs_dyn.npz": [
        {},
        {},
        dict(L8="2.0e-5 0.0 0.0", L21="2.0e-3", L20="0.5"),
        dict(L8="2.0e-5 0.0 0.0", L21="2.0e-3", L20="0.5", L27=25, L23="1500.0", L39="0.9 0.02", L31=50),
        dict(L8="2.0e-5 0.0 0.0", L21="2.0e-3", L20="0.5", L27=25, L23="1500.0", L39="0.9 0.02", L31=50,
             L4=350, L29=50),
    ],
}


# Seed of oracle/mpishim/seeded_rand.h (LBM_FIXTURE_SEED): the colour-gradient
# program built with it draws the random numbers that lbm_cg --seed draws.
FIXTURE_SEED = 20261203

# Runs of the seeded program build (ref_cg3_main_seeded): random initial
# phase and random phase faces; name -> INPUT overrides.
CG_SEEDED_RUNS = {
    # random initial phase at ini_Sat = 0.45, random phase faces (flag 3) on
    # x+ and y+, the initial phase on x-; phase VTK every 50 steps
    "cg_outputs_rand.npz": dict(L7=1, L15="3 1", L16="3 0", L37=0.45, L29=-1, L30=-1, L45=0),
    # random initial phase at ini_Sat = 0.6 with a partial window 3..10 on x
    # and buffer phase +1 outside it (the sums limited to the window)
    "cg_outputs_rand_buf.npz": dict(L37=0.6, L38=1, L40="1 0 0", L41="10 3", L29=-1, L30=-1, L45=0),
    # imbibition control over 50 target saturations with random phase faces
    # on both x faces (ini_Sat 0.9, random initial phase): the targets passed
    # at the reports of steps 10, 20, 30 write the phase field and move the
    # faces' threshold; reports every 10 steps
    "cg_outputs_imb.npz": dict(L64="1 50", L7=1, L15="3 3", L37=0.9, L27=10, L29=-1, L30=-1, L45=0),
    # drainage control, the phase faces turned on by the control itself
    # (in_psi_BC = 0 in the file), ini_Sat 0.1
    "cg_outputs_drain.npz": dict(L64="2 50", L7=0, L15="3 3", L37=0.1, L27=10, L29=-1, L30=-1, L45=0),
}


def run_cg_program(workdir, input_txt, mask, psi, args=(), seeded=False, versions=None):
    """versions: the texts the k-th opening of INPUT.dat reads (a named pipe,
    tests/helpers.py InputVersions), for a run with input_dynamic."""
    import subprocess

    exe = os.path.join(ROOT, "oracle", "_ref", "ref_cg3_main_seeded" if seeded else "ref_cg3_main")
    G.write_ascii(os.path.join(workdir, "mask.dat"), mask)
    with open(os.path.join(workdir, "phase.dat"), "w") as f:
        f.write(phase_text(psi))
    if versions is None:
        with open(os.path.join(workdir, "INPUT.dat"), "w") as f:
            f.write(input_txt)
        subprocess.run([exe, "INPUT.dat", *args], cwd=workdir, check=True, capture_output=True)
        return
    from helpers import InputVersions

    with InputVersions(os.path.join(workdir, "INPUT.dat"), versions) as iv:
        subprocess.run([exe, "INPUT.dat", *args], cwd=workdir, check=True, capture_output=True, timeout=600)
        print("input openings served:", iv.served)


def collect_cg(workdir, prefix, fg_width=7):
    out = {}
    for name in sorted(os.listdir(workdir)):
        if not name.startswith(prefix):
            continue
        key = name[len(prefix):]
        data = open(os.path.join(workdir, name), "rb").read()
        if key.startswith("LBM_checkpoint_"):
            width = {"rho": 1, "velocity": 3, "f": 19, "psi": 1, "rhor": 1, "rhob": 1, "fg": fg_width}[key.split("_")[2]]
            out[key] = digest(np.frombuffer(data, dtype=np.float64).reshape(-1, width)[1:])
        else:
            out[key] = data
    return out


def save_cg(fname, mask, psi, input_txt, files, seed=None, versions=None):
    blob = {"mask": pack(mask), "shape": np.array(mask.shape), "phase": np.frombuffer(phase_text(psi).encode(), np.uint8),
            "input": np.frombuffer(input_txt.encode(), np.uint8), "names": np.array(sorted(files))}
    if seed is not None:
        blob["seed"] = np.array(seed, dtype=np.uint64)
    for k, v in enumerate(versions or ()):
        blob[f"input_version_{k}"] = np.frombuffer(v.encode(), np.uint8)
    for k, v in files.items():
        blob[k] = np.frombuffer(v, np.uint8) if isinstance(v, bytes) else np.array(v)
    np.savez_compressed(os.path.join(HERE, fname), **blob)
    print(fname, sorted(files))


def cg_program_outputs(only=None):
    """Every file the colour-gradient program writes for the runs of CG_RUNS
    (those whose name contains `only`, when given), and two restarts: the
    step-100 checkpoint of cg_outputs / cg_outputs_pre1 read back
    (mode_backup_ini = 100, prefix ./out_) and run for 60 more steps
    (cg_outputs_restart.npz / cg_outputs_pre1_restart.npz, files prefixed
    rst_)."""
    import tempfile

    mask, psi = cg_geometry()
    for fname, kv in CG_RUNS.items():
        if only and only not in fname:
            continue
        text = cg_input_text(**kv)
        with tempfile.TemporaryDirectory() as d:
            run_cg_program(d, text, mask, psi)
            files = collect_cg(d, "out_")
            if fname == "cg_outputs.npz":
                rst = cg_input_text(L4=59, L27=20, L29=-1, L30=-1, L31=40, L34="./rst_", L45=0, L46=100)
                run_cg_program(d, rst, mask, psi, ("./out_",))
                save_cg("cg_outputs_restart.npz", mask, psi, rst, collect_cg(d, "rst_"))
            if fname == "cg_outputs_pre1.npz":
                rst = cg_input_text(**{**kv, "L4": 59, "L27": 20, "L31": 40, "L34": "./rst_", "L45": 0,
                                       "L46": 100})
                run_cg_program(d, rst, mask, psi, ("./out_",))
                save_cg("cg_outputs_pre1_restart.npz", mask, psi, rst, collect_cg(d, "rst_"))
        save_cg(fname, mask, psi, text, files)
    for fname, kv in CG_SEEDED_RUNS.items():
        if only and only not in fname:
            continue
        text = cg_input_text(**kv)
        with tempfile.TemporaryDirectory() as d:
            run_cg_program(d, text, mask, psi, seeded=True)
            files = collect_cg(d, "out_")
        save_cg(fname, mask, psi, text, files, seed=FIXTURE_SEED)
    for fname, steps in CG_DYNAMIC_RUNS.items():
        if only and only not in fname:
            continue
        texts = [cg_input_text(**{**CG_DYNAMIC_BASE, **kv}) for kv in steps]
        with tempfile.TemporaryDirectory() as d:
            run_cg_program(d, texts[0], mask, psi, versions=texts)
            files = collect_cg(d, "out_")
        save_cg(fname, mask, psi, texts[0], files, versions=texts)
    for fname, (geometry, kv) in CG_GEOMETRY_RUNS.items():
        if only and only not in fname:
            continue
        gmask, gpsi = geometry()
        text = cg_input_text(**kv)
        with tempfile.TemporaryDirectory() as d:
            run_cg_program(d, text, gmask, gpsi)
            files = collect_cg(d, "out_")
        save_cg(fname, gmask, gpsi, text, files)


def bc_cases():
    """(name, Boundaries, g, perdir) of the boundary-condition fixture: for
    each Sub_BC 0..3, pressure on the two x faces, pressure on all six faces
    with a body force, velocity on all six faces, and pressure on y with
    velocity on x+ and z-."""
    B = oracle.Boundaries
    out = []
    for sb in range(4):
        out.append((f"pre_x_{sb}", B(sub_bc=sb, in_bc=1, pre=(1, 1, 0, 0, 0, 0), p=(1.0, 1.01, 1, 1, 1, 1)),
                    (0.0, 0.0, 0.0), 1))
        out.append((f"pre_all_{sb}", B(sub_bc=sb, in_bc=1, pre=(1,) * 6, p=(1.0, 1.01, 1.002, 0.999, 1.003, 1.001)),
                    (1e-5, 0.0, 0.0), 1))
        out.append((f"vel_all_{sb}", B(sub_bc=sb, in_bc=0, vel=(1,) * 6, v=(0.01, 0.01, 0.002, -0.003, 0.001, 0.004)),
                    (1e-5, 0.0, 0.0), 1))
        out.append((f"mix_{sb}", B(sub_bc=sb, in_bc=1, pre=(0, 0, 1, 1, 0, 0), p=(1, 1, 1.0, 1.01, 1, 1),
                                   vel=(1, 0, 0, 0, 0, 1), v=(0.01, 0.02, 0, 0, 0.003, 0.004)), (0.0, 0.0, 0.0), 2))
    return out


BC_SHAPE, BC_SEED, BC_NU, BC_STEPS = (14, 8, 10), 11, 0.1, 21


def bc_fixture():
    """Pressure/velocity boundaries: the reference (boundary_pressure,
    boundary_velocity at one rank) on 14x8x10 spheres, 21 steps per case: the
    face lists, SHA-256 of f, u, rho (rows 1..) and Comput_Perm's output."""
    mask = G.overlapping_spheres(BC_SHAPE, 0.6, 2.5, seed=BC_SEED)
    ref = oracle.ReferenceSP3()
    blob = {"mask": pack(mask), "shape": np.array(mask.shape), "nu": BC_NU, "steps": BC_STEPS}
    for name, bc, g, perdir in bc_cases():
        ref.set_boundaries(bc, perdir)
        ref.create(mask, BC_NU, g)
        if name == "pre_x_0":
            for fc in range(6):
                blob[f"face_{fc}"] = ref.face_list(fc)
        ref.step(BC_STEPS)
        f, u, rho = ref.fields()
        e, perm, ua = ref.perm()
        blob[name] = np.array([digest(f[1:]), digest(u[1:]), digest(rho[1:])])
        blob[name + ":perm"] = np.array([*perm, ua])
    ref.set_boundaries(None)
    np.savez_compressed(os.path.join(HERE, "sp_bc.npz"), **blob)
    print("sp_bc", len(bc_cases()), "cases")


ST7_SHAPE, ST7_SEED, ST7_D, ST7_NRANKS = (16, 10, 8), 41, 0.005, 2


def solute_input(**kv):
    """INPUT file of the solute program: the reference's sample
    Single_Phase_3D/INPUT_SOLUTE.dat (its first 51 lines, read at run time)
    with some values replaced; keys are the 0-based line numbers."""
    lines = open(os.path.join(oracle.REFERENCE_ROOT, "Single_Phase_3D", "INPUT_SOLUTE.dat")).read().splitlines()[:51]
    for i, v in kv.items():
        lines[int(i[1:])] = f"{v}\t\t:{lines[int(i[1:])].split(':', 1)[1]}"
    return "\n".join(lines) + "\n"


def st7_fixture(out=None, program="ref_st7_slab"):
    """The reference's own slab programs at two ranks (multi-process MPI
    stand-in): the slab single-phase program makes the flow of a 16x10x8
    sphere pack and writes Velocity_for_solute_100.<rank>.bin; the solute
    program (D = 0.005, initial concentration uniform in [0, 1) as float)
    advects and diffuses for 61 steps and backs up the concentration every 20
    steps.  Stored: mask, initial concentration, the velocity records (slab
    order, ranks concatenated), rank sizes, and the concentration at steps
    20, 40, 60 (slab order).  program = "ref_st19_slab" runs the D3Q19
    solute program on the same inputs instead (st19_slab.npz)."""
    import tempfile

    sp, st = oracle.slab_program("ref_sp_slab"), oracle.slab_program(program)
    if not (sp and st):
        raise SystemExit(f"oracle/_ref/ref_sp_slab and {program} are needed (make -C oracle ref)")
    mask = G.overlapping_spheres(ST7_SHAPE, 0.6, 2.5, seed=ST7_SEED)
    nx, ny, nz = ST7_SHAPE
    c0 = np.random.default_rng(5).uniform(0, 1, mask.shape).astype(np.float32)
    with tempfile.TemporaryDirectory() as d:
        G.write_ascii(os.path.join(d, "mask.dat"), mask)
        flow = input_text(L1="mask.dat", L2=f"{nx} {ny} {nz}", L3=100, L18=50, L20=-1, L21=-1, L24="./", L32=-1,
                          L34=100)
        open(os.path.join(d, "INPUT.dat"), "w").write(flow)
        assert oracle.run_ranks(sp, ["INPUT.dat"], ST7_NRANKS, d) == [0] * ST7_NRANKS
        with open(os.path.join(d, "phase.dat"), "w") as fh:
            fh.write("\n".join(repr(float(v)) for v in c0.reshape(-1)) + "\n")
        text = solute_input(L1="mask.dat", L2="phase.dat", L3=f"{nx} {ny} {nz}", L4=60, L23=ST7_D, L28=20,
                            L33="0 1000", L36="./st_", L45=20, L47=100)
        open(os.path.join(d, "INPUT_st.dat"), "w").write(text)
        assert oracle.run_ranks(st, ["INPUT_st.dat"], ST7_NRANKS, d) == [0] * ST7_NRANKS
        vel = [np.fromfile(os.path.join(d, f"Velocity_for_solute_100.{r}.bin")) for r in range(ST7_NRANKS)]
        conc = {m: np.concatenate([np.fromfile(os.path.join(d, f"st_LBM_checkpoint_psi_{m}.{r}.bin_input"))[1:]
                                   for r in range(ST7_NRANKS)]) for m in (20, 40, 60)}
    np.savez_compressed(out or os.path.join(HERE, "st7_slab.npz"), mask=pack(mask), shape=np.array(mask.shape), c0=c0,
                        diffusivity=ST7_D, nranks=ST7_NRANKS, u_slab=np.concatenate(vel),
                        rank_nodes=np.array([v.size // 3 for v in vel]), steps=np.array([20, 40, 60]),
                        c20=conc[20], c40=conc[40], c60=conc[60], input_solute=np.frombuffer(text.encode(), np.uint8))
    print("st7_slab", mask.shape, [v.size // 3 for v in vel])


def st7_program_outputs(program="ref_st7_slab", tag="st7", variants=True, only=None):
    """The solute program itself at two ranks (multi-process MPI stand-in):
    every file it writes, for the drop-in driver's byte-for-byte test.  The
    slab single-phase program first makes the flow of the st7_slab geometry
    (Velocity_for_solute_100.<rank>.bin, stored verbatim); then the solute
    program runs 61 steps with reports every 20, velocity VTK every 40,
    concentration VTK every 20, checkpoints every 40, solids written as 0.5,
    in both output layouts (Out_Mode 1: st7_outputs.npz, Out_Mode 0:
    st7_outputs_b.npz), with the dispersion statistics along x
    (st7_outputs_dis.npz) and along z with a y window (st7_outputs_dis3.npz);
    and a restart from the step-40 checkpoint (copied to
    the unprefixed names Backup_init reads) runs 31 more steps
    (st7_outputs_restart.npz).  program = "ref_st19_slab", tag = "st19",
    variants = False: the D3Q19 solute program, Out_Mode 1 run and restart
    only (st19_outputs.npz, st19_outputs_restart.npz)."""
    import shutil
    import tempfile

    sp, st = oracle.slab_program("ref_sp_slab"), oracle.slab_program(program)
    if not (sp and st):
        raise SystemExit(f"oracle/_ref/ref_sp_slab and {program} are needed (make -C oracle ref)")
    mask = G.overlapping_spheres(ST7_SHAPE, 0.6, 2.5, seed=ST7_SEED)
    nx, ny, nz = ST7_SHAPE
    c0 = np.random.default_rng(5).uniform(0, 1, mask.shape).astype(np.float32)
    phase = "\n".join(repr(float(v)) for v in c0.reshape(-1)) + "\n"
    with tempfile.TemporaryDirectory() as d:
        G.write_ascii(os.path.join(d, "mask.dat"), mask)
        flow = input_text(L1="mask.dat", L2=f"{nx} {ny} {nz}", L3=100, L18=50, L20=-1, L21=-1, L24="./", L32=-1,
                          L34=100)
        open(os.path.join(d, "INPUT.dat"), "w").write(flow)
        assert oracle.run_ranks(sp, ["INPUT.dat"], ST7_NRANKS, d) == [0] * ST7_NRANKS
        vel = {f"Velocity_for_solute_100.{r}.bin": open(os.path.join(d, f"Velocity_for_solute_100.{r}.bin"), "rb").read()
               for r in range(ST7_NRANKS)}
        open(os.path.join(d, "phase.dat"), "w").write(phase)
        # dispersion statistics along x every 20 steps (written after step 10)
        # and along z every 40, both layouts of the run above
        runs = {f"{tag}_outputs.npz": ("./st_", dict(L29=1)),
                # self-defined lattice velocity dx = 1, dt = 2 (tau_s, the
                # report's Peclet and Courant numbers, the dispersion
                # statistics along x every 20 steps; for D3Q19 also the
                # equilibrium's divisions by lat_c^2, lat_c^4)
                f"{tag}_outputs_lat.npz": ("./sl_", dict(L29=1, L33="1 20", L35="1 1.0 2.0"))}
        if variants:
            runs.update({"st7_outputs_b.npz": ("./sb_", dict(L29=0)),
                         "st7_outputs_dis.npz": ("./sd_", dict(L29=1, L33="1 20", L39=10)),
                         "st7_outputs_dis3.npz": ("./sz_", dict(L29=0, L33="3 40", L39=-1, L40="0 1 0",
                                                                 L42="8 2"))})
        for fname, (prefix, kv) in runs.items():
            if only and only not in fname:
                continue
            base = dict(L1="mask.dat", L2="phase.dat", L3=f"{nx} {ny} {nz}", L4=60, L7="0.0 0.5", L23=ST7_D,
                        L28=20, L30=40, L32=20, L33="0 1000", L36=prefix, L45=40, L47=100)
            base.update(kv)
            text = solute_input(**base)
            open(os.path.join(d, "INPUT_st.dat"), "w").write(text)
            assert oracle.run_ranks(st, ["INPUT_st.dat"], ST7_NRANKS, d) == [0] * ST7_NRANKS
            save_st7(fname, mask, phase, text, vel, collect_cg(d, prefix[2:], fg_width=19 if tag == "st19" else 7))
        if only and only not in f"{tag}_outputs_restart.npz":
            return
        for r in range(ST7_NRANKS):
            for what in ("psi", "fg"):
                shutil.copy(os.path.join(d, f"st_LBM_checkpoint_{what}_40.{r}.bin_input"),
                            os.path.join(d, f"LBM_checkpoint_{what}_40.{r}.bin_input"))
        text = solute_input(L1="mask.dat", L2="phase.dat", L3=f"{nx} {ny} {nz}", L4=30, L7="0.0 0.5", L23=ST7_D,
                            L28=10, L29=1, L30=-1, L32=30, L33="0 1000", L36="./rs_", L45=-1, L46=40, L47=100)
        open(os.path.join(d, "INPUT_st.dat"), "w").write(text)
        assert oracle.run_ranks(st, ["INPUT_st.dat"], ST7_NRANKS, d) == [0] * ST7_NRANKS
        save_st7(f"{tag}_outputs_restart.npz", mask, phase, text, vel,
                 collect_cg(d, "rs_", fg_width=19 if tag == "st19" else 7))


def save_st7(fname, mask, phase, text, vel, files):
    blob = {"mask": pack(mask), "shape": np.array(mask.shape), "phase": np.frombuffer(phase.encode(), np.uint8),
            "input": np.frombuffer(text.encode(), np.uint8), "nranks": ST7_NRANKS,
            "names": np.array(sorted(files)), "velocity_files": np.array(sorted(vel))}
    for k, v in vel.items():
        blob["file:" + k] = np.frombuffer(v, np.uint8)
    for k, v in files.items():
        blob[k] = np.frombuffer(v, np.uint8) if isinstance(v, bytes) else np.array(v)
    np.savez_compressed(os.path.join(HERE, fname), **blob)
    print(fname, sorted(files))


SLAB_GROUPS = dict(n_sub=[1, 2, 0, 0], size=[8, 4, 1, 1], corner=[0, 0, 0, 2, 2, 1, 0, 0, 0, 0, 0, 0])


def slab_perm_fixture(out=None):
    """The slab single-phase program at two ranks on the sp_outputs mask with
    its sub-volume permeabilities on: Comput_Perm_LOCAL every report
    (loc_perm = 1) and Comput_Grop_Perm every 50 steps (divisions: one cube of
    8 at (0,0,0), 2^3 cubes of 4 from (2,2,1)); 101 steps.  Stored: the INPUT
    file, mask, Results.txt and the Perm_<size>.output files."""
    import tempfile

    sp = oracle.slab_program("ref_sp_slab")
    if not sp:
        raise SystemExit("oracle/_ref/ref_sp_slab is needed (make -C oracle ref)")
    mask = G.overlapping_spheres((14, 12, 10), 0.6, 2.5, seed=21)
    g = SLAB_GROUPS
    corners = [" ".join(str(c) for c in g["corner"][3 * i:3 * i + 3]) for i in range(4)]
    text = input_text(L1="mask.dat", L2="14 12 10", L3=100, L17=1, L18=50, L20=-1, L21=-1, L24="./out_", L26=1,
                      L32=-1, L34=-1, L36=50, L37=" ".join(map(str, g["n_sub"])), L38=" ".join(map(str, g["size"])),
                      L39=corners[0], L40=corners[1], L41=corners[2], L42=corners[3])
    with tempfile.TemporaryDirectory() as d:
        G.write_ascii(os.path.join(d, "mask.dat"), mask)
        open(os.path.join(d, "INPUT.dat"), "w").write(text)
        assert oracle.run_ranks(sp, ["INPUT.dat"], 2, d) == [0, 0]
        files = {n[len("out_"):]: open(os.path.join(d, n), "rb").read() for n in sorted(os.listdir(d))
                 if n.startswith("out_") and (n.endswith(".output") or n.endswith("Results.txt"))}
    blob = {"mask": pack(mask), "shape": np.array(mask.shape), "input": np.frombuffer(text.encode(), np.uint8),
            "names": np.array(sorted(files))}
    for k, v in files.items():
        blob[k] = np.frombuffer(v, np.uint8)
    np.savez_compressed(out or os.path.join(HERE, "sp_slab_perm.npz"), **blob)
    print("sp_slab_perm", sorted(files))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--bc", action="store_true")
    ap.add_argument("--st7", action="store_true")
    ap.add_argument("--slab-perm", action="store_true")
    ap.add_argument("--cfg1", action="store_true")
    ap.add_argument("--cg", action="store_true")
    ap.add_argument("--outputs", action="store_true")
    ap.add_argument("--cg-outputs", action="store_true")
    ap.add_argument("--only", default=None,
                    help="--outputs / --cg-outputs / --st7-outputs / --st19: runs whose fixture name contains this")
    ap.add_argument("--st7-outputs", action="store_true")
    ap.add_argument("--st19", action="store_true", help="D3Q19 solute program fixtures")
    a = ap.parse_args()
    oracle.build()
    if a.st7_outputs:
        st7_program_outputs(only=a.only)
        return
    if a.st19:
        if not a.only:
            st7_fixture(os.path.join(HERE, "st19_slab.npz"), program="ref_st19_slab")
        st7_program_outputs(program="ref_st19_slab", tag="st19", variants=False, only=a.only)
        return
    if a.cg_outputs:
        cg_program_outputs(a.only)
        return
    if a.cg:
        cg_small()
        return
    if a.outputs:
        program_outputs(a.only)
        return
    if a.bc:
        bc_fixture()
        return
    if a.st7:
        st7_fixture()
        return
    if a.slab_perm:
        slab_perm_fixture()
        return
    ref = oracle.ReferenceSP3()
    if a.cfg1:
        cfg1(ref)
    else:
        small(ref)
        mid(ref)


if __name__ == "__main__":
    main()
