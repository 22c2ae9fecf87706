/*
 * lbm.h -- C ABI of liblbm.so, a B200 (sm_100a) implementation of the sparse
 * D3Q19 MRT lattice Boltzmann update of the jianhui-lbm suite.
 *
 * The reference exposes no library API: each solver is one C++ program whose
 * hot path is a pair of void functions over globals.  Every entry point below
 * states which reference code it replaces (paths relative to the reference
 * project root).  Abbreviations:
 *   SP  = Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars.cpp
 *   SP3 = Single_Phase_3D/SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp
 *   CG3 = MP_3D/Multi_Component_CG_MPI_SPARSE_Software_3DPartition.cpp
 *   CG  = MP_3D/Multi_Component_CG_MPI_SPARSE_Software.cpp
 *   ST7 = Single_Phase_3D/Solute_Transport_MPI_Software_Spars_6V.cpp
 *
 * Conventions
 *   - Status: every function returns lbm_status (0 = OK, negative = error);
 *     lbm_last_error() gives the message of the last failure on that thread.
 *     Nothing calls exit() (the reference exits on a missing geometry file,
 *     SP3:941-949).
 *   - Ownership: a handle owns all device memory it allocates; caller buffers
 *     are host memory and are copied synchronously.
 *   - Node ids and layouts in and out of the library are the reference's:
 *     fluid ids are 1-based in SP3 compaction order, row 0 is an unused dummy
 *     row; populations are AoS double[(count+1)*19]; velocity double[(count+1)*3].
 *   - Masks are uint8 [nz][ny][nx] (x fastest), 0 = pore, non-zero = solid,
 *     the token order of the reference's ASCII geometry file.
 *   - Threading: one handle is used by one host thread at a time and runs on
 *     its own CUDA stream; distinct handles may run concurrently.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

typedef int lbm_status;
enum {
  LBM_OK = 0,
  LBM_ERR_ARG = -1,            /* invalid argument or size */
  LBM_ERR_IO = -2,             /* file missing / unreadable / short */
  LBM_ERR_OOM = -3,            /* device or host allocation failed */
  LBM_ERR_CUDA = -4,           /* CUDA runtime error */
  LBM_ERR_NAN = -5,            /* non-finite velocity detected (SP3:733) */
  LBM_ERR_NOT_CONVERGED = -6,  /* step cap reached before the tolerance */
  LBM_ERR_FORMAT = -7,         /* malformed INPUT*.dat or geometry */
  LBM_ERR_STATE = -8,          /* call not valid in the handle's state */
  LBM_ERR_OVERSPEED = -9,      /* u_max >= 10 five times (SP3:722, 734) */
  LBM_ERR_NO_DEVICE = -10      /* no CUDA device / kernel image */
};

typedef enum {
  LBM_PREC_F64 = 0,       /* FP64, bit-exact with the reference's collision */
  LBM_PREC_F32 = 1,       /* FP32 deviation storage f_i - w_i, FP32 math */
  LBM_PREC_F16 = 2,       /* FP16 scaled-deviation storage, FP32 math */
  LBM_PREC_F64_FAST = 3   /* FP64 deviation storage, sparse FMA moments */
} lbm_precision;

typedef enum {
  LBM_ORDER_REFERENCE = 0, /* SP3 compaction order (x fastest) */
  LBM_ORDER_MORTON = 1,    /* Z-order curve over (x,y,z) */
  LBM_ORDER_HILBERT = 2,   /* 3-D Hilbert curve */
  LBM_ORDER_BRICK = 3,     /* 16x4x4 bricks, x fastest inside, bricks x fastest */
  LBM_ORDER_AUTO = -1      /* picked by lbm_autotune */
} lbm_ordering;

/* Pressure / velocity boundaries (INPUT.dat lines SP3:299-305, 318;
 * boundary_pressure SP3:2656-3116, boundary_velocity SP3:2450-2655).  Faces
 * in INPUT.dat order: xp (x = nx-1), xn (x = 0), yp, yn, zp, zn.  A face with
 * pressure[i] == 1 or velocity[i] == 1 overwrites the post-streaming
 * populations of its pore nodes every step, by the Sub_BC rule:
 *   pressure 0: f_eq(rho_b, 0);  1: f_eq(rho_b, u of the inward neighbour);
 *            2: moments of the inward neighbour with rho replaced by rho_b;
 *            3: f_eq(rho_b, u_nb) + (f - f_eq) of the -y neighbour;
 *   velocity 0, 1: f_eq(1, u_b);  2: non-equilibrium bounce-back of the
 *            incoming directions (x flags act on the z faces and z flags on
 *            the x faces, as in the reference);  3: f_eq(rho of the inward
 *            neighbour, u_b).
 * in_bc = 1 adds |p_+ - p_-| c_s^2 / L to the force in Comput_Perm. */
typedef struct lbm_boundary {
  int sub_bc;        /* Sub_BC 0..3 */
  int in_bc;         /* in_BC */
  int pressure[6];   /* pre_xp, pre_xn, pre_yp, pre_yn, pre_zp, pre_zn */
  double rho[6];     /* p_xp .. p_zn: boundary density */
  int velocity[6];   /* vel_xp .. vel_zn */
  double vel[6];     /* v_xp .. v_zn: normal velocity of the face */
} lbm_boundary;

/* Run parameters of the single-phase solver (the physics subset of INPUT.dat,
 * SP3:283-338).  lbm_params_default() fills reference defaults. */
typedef struct lbm_params {
  double nu;          /* kinematic viscosity in_vis; tau = 3 nu + 0.5 (SP3:1289-1296) */
  double gx, gy, gz;  /* body force as acceleration (SP3:1423-1500) */
  double u_init[3];   /* initial velocity inivx..inivz (SP3:1331-1333) */
  int precision;      /* lbm_precision */
  int ordering;       /* lbm_ordering (LBM_ORDER_AUTO allowed) */
  int block_size;     /* threads per block; 0 = default, autotune may change */
  int perdir;         /* PerDir 1..3: permeability direction (SP3:3560-3570) */
  int window[6];      /* per_xn,per_xp,per_yn,per_yp,per_zn,per_zp; all -1 = whole box */
  double fp16_scale;  /* LBM_PREC_F16 storage scale; 0 = derived from nu and |g| */
  int device;         /* CUDA device ordinal */
  lbm_boundary bc;    /* pressure/velocity boundaries; all faces off by default (fully periodic) */
} lbm_params;

/* Diagnostics of one reporting step: Error (SP3:3118-3196) and
 * Comput_Perm (SP3:3518-3648) at the current state. */
typedef struct lbm_diag {
  long long step;        /* time steps completed */
  double perm[3];        /* Q_d / V * nu / g_d (lattice units) */
  double perm_rel_change;/* (k - k_prev)/k_prev along perdir */
  double u_ave;          /* |Q| / (V * porosity) -- the convergence quantity */
  double u_max;          /* max |u| over nodes 1..count-1 */
  double u_rel_change;   /* ||u - u_prev|| / ||u|| over nodes 1..count-1 */
  double u_mean_speed;   /* sum |u| / (V * porosity) over nodes 1..count-1 */
  double mass;           /* sum rho over all fluid nodes */
  double porosity;       /* pore fraction of the window */
  int nan_detected;      /* 1 when u_rel_change is NaN (SP3:733) */
  int converged;         /* set by lbm_run_to_convergence */
} lbm_diag;

typedef struct lbm_handle lbm_handle;

/* ---------------------------------------------------------------- basics */
LBM_API const char* lbm_last_error(void);
LBM_API const char* lbm_status_string(lbm_status s);
LBM_API int lbm_abi_version(void);
LBM_API void lbm_params_default(lbm_params* p);

/* ------------------------------------------------- input formats (SP3 L0/L1) */

/* The INPUT.dat / INPUT_Partition.dat parameter file of the single-phase
 * solvers, every field in the file's line order (SP3:283-340: one value group
 * per line followed by a comment; NX..NZ stored as given, not minus one). */
typedef struct lbm_input {
  char geometry_file[128];
  int nx, ny, nz;
  int n_max;
  double reso;
  int in_bc;
  double gx, gy, gz;
  int pre_xp; double p_xp; int pre_xn; double p_xn;
  int pre_yp; double p_yp; int pre_yn; double p_yn;
  int pre_zp; double p_zp; int pre_zn; double p_zn;
  int vel_xp; double v_xp; int vel_xn; double v_xn;
  int vel_yp; double v_yp; int vel_yn; double v_yn;
  int vel_zp; double v_zp; int vel_zn; double v_zn;
  double in_vis;
  double inivx, inivy, inivz;
  int wr_per, perdir, fre_re, out_mode, fre_ve, fre_de;
  int lattice_v; double dx_input, dt_input;
  char output_path[128];
  int sub_bc, loc_perm;
  int par_per_x, par_per_y, par_per_z;
  int per_xp, per_xn, per_yp, per_yn, per_zp, per_zn;
  int fre_backup, mode_backup_ini, vel_sol;
  int gperm, n_gperm[4], size_gperm[4], c_gperm[4][3];
  int decbin;
  int nnf_module; double nnf_m, nnf_n;
} lbm_input;

/* Parses a single-phase INPUT file (replaces the rank-0 reader SP3:283-340). */
LBM_API lbm_status lbm_read_input(const char* path, lbm_input* out);

/* Reads a geometry file into a uint8 [nz][ny][nx] mask (0 pore, 1 solid).
 * decbin 0: ASCII tokens in x-fastest order, non-zero = solid (SP3:929-943);
 * decbin 1: int32 C-order [i][j][k] (SP3:947-961). */
LBM_API lbm_status lbm_read_mask(const char* path, int nx, int ny, int nz, int decbin, uint8_t* mask_out);

/* ------------------------------------------------ single-phase solver (SP3) */

/* Builds the fluid-node compaction (SP3:1018-1071), the pull neighbour table
 * with halfway bounce-back resolved (equivalent of nei_loc, SP3:1099-1151),
 * the MRT constants (Comput_MI SP3:838, init SP3:1278) and the device state.
 * The mask is copied; the caller keeps ownership.  The first creation on a
 * device also pins 32 MiB of host memory for the process's field and
 * population reads (shared by every handle, kept until the process ends). */
LBM_API lbm_status lbm_create(const lbm_params* p, const uint8_t* mask, int nx, int ny, int nz,
                      lbm_handle** out);

/* Reads INPUT.dat and its geometry file and creates the solver (main SP3:258-555
 * at one rank), pressure/velocity faces (pre_*, vel_*, Sub_BC) included, and
 * a self-defined lattice velocity (lattice_v = 1 with dx, dt: lbm_set_lattice).
 * The non-Newtonian module returns LBM_ERR_ARG. */
LBM_API lbm_status lbm_create_from_input(const char* input_path, int precision, int ordering,
                                 lbm_handle** out, lbm_input* parsed_out);

/* Self-defined lattice velocity (lattice_v with dx, dt; SP3:1286-1296,
 * 1326-1330): lat_c = dx/dt, c_s^2 = lat_c^2 / 3, tau = nu / (c_s^2 dt) + 1/2;
 * the discrete velocities are e lat_c in the equilibrium (divided by
 * c2 = lat_c^2 and c4 = c2^2), the Guo force and the macro step, the force
 * enters the moments as dt F and the velocity as dt g / 2, the face rules'
 * equilibria use the same feq, and the pressure term of the permeability uses
 * c_s^2 and dx.  Velocities in and out (fields, reductions, checkpoints, face
 * velocities) are the velocity itself.  LBM_PREC_F64 reproduces the
 * reference's arithmetic bit for bit; the other precisions step in units of
 * lat_c.  Call after lbm_create and before the first step: the state restarts
 * from the initial equilibrium on the new lattice.  The default lattice is
 * dx = dt = 1. */
LBM_API lbm_status lbm_set_lattice(lbm_handle* h, double dx, double dt);

LBM_API void lbm_destroy(lbm_handle* h);

/* Advances nsteps time steps: each is collision (SP3:1398-1819) + streaming +
 * comput_macro_variables (SP3:2401-2446), fused into one kernel per step. */
LBM_API lbm_status lbm_step(lbm_handle* h, int nsteps);

/* Diagnostics at the current state (Error + Comput_Perm, SP3:712-713).  The
 * velocity change is measured against the velocity one step earlier, exactly
 * like the reference's u0 (comput_macro_variables saves u0 every step). */
LBM_API lbm_status lbm_reduce(lbm_handle* h, lbm_diag* out);

/* Runs until |(u_ave_prev - u_ave)/u_ave_prev| < tol at a check every
 * check_every steps (the SP stop test SP:812-816, u_ave from Comput_Perm),
 * or max_steps.  Returns LBM_OK when converged, LBM_ERR_NOT_CONVERGED at the
 * cap, LBM_ERR_NAN / LBM_ERR_OVERSPEED on the reference's stop conditions. */
LBM_API lbm_status lbm_run_to_convergence(lbm_handle* h, double tol, int check_every, int max_steps,
                                  lbm_diag* out);

/* Sub-volume flux sums of the current state: for each box (xn, xp, yn, yp,
 * zn, zp inclusive, clipped to the grid) the sums of u_x, u_y, u_z over its
 * pore cells and the number of pore cells, out[4*b .. 4*b+3].  The flux sums
 * of Comput_Perm's window (SP3:3559-3590), Comput_Grop_Perm's cubes
 * (SP:4886-5091) and Comput_Perm_LOCAL's plane (SP:4831-4884).  Sums run in
 * a fixed order on the device (reproducible, not the reference's order). */
LBM_API lbm_status lbm_box_sums(lbm_handle* h, int nbox, const int32_t* boxes, double* out);

/* Comput_Grop_Perm (SP:4886-5091): division d has n_sub[d]^3 cubes of edge
 * size[d], the first with low corner corner[3d .. 3d+2]; cube (a, b, c), in
 * the reference's loop order (a = x outer, c = z inner), starts at corner +
 * (a, b, c) * size[d].  out[4*cube ..] = permeability (x, y, z; lattice
 * units: Q / size^3 * nu / (g + dp)) and porosity (pores / size^3).  dp uses
 * the whole box length (SP:4928-4941). */
LBM_API lbm_status lbm_group_perm(lbm_handle* h, int ndiv, const int* n_sub, const int* size, const int* corner,
                                  double* out);

/* Comput_Perm_LOCAL (SP:4831-4884): permeability from the flux through the
 * plane x = nx-2, normalised by the window's cross-sections. */
LBM_API lbm_status lbm_local_perm(lbm_handle* h, double perm[3]);

/* Number of fluid nodes (the reference's Count) and geometry facts. */
LBM_API lbm_status lbm_info(lbm_handle* h, int* count, double* porosity, long long* step);

/* rho[(count+1)] and u[(count+1)*3] in reference id order (row 0 zero);
 * either pointer may be NULL.  Same values comput_macro_variables leaves in
 * the reference's rho/u arrays.  Large host arrays are filled from pinned
 * staging by several threads, and transparent huge pages are requested for
 * them (madvise; their contents are not otherwise touched). */
LBM_API lbm_status lbm_get_fields(lbm_handle* h, double* rho, double* u);

/* Post-streaming populations f[(count+1)*19], reference id order -- the
 * reference's f array after comput_macro_variables. */
LBM_API lbm_status lbm_get_populations(lbm_handle* h, double* f);

/* Replaces the state (the reference's Backup_init, SP3:3652-3767): rho, u and
 * f in reference layout.  The next step uses rho and u as given, like the
 * reference's first collision after init or a restart. */
LBM_API lbm_status lbm_set_state(lbm_handle* h, const double* rho, const double* u, const double* f);

/* coor[(count+1)] = i*ny*nz + j*nz + k per fluid id (SP3:1065-1071). */
LBM_API lbm_status lbm_export_compaction(lbm_handle* h, int32_t* coor);

/* The neighbour table in the reference's push form nei_loc[(count+1)*19]
 * (SP3:1099-1151: destination id, 0 = bounce-back), reconstructed from the
 * device pull table -- for the bit-exact table test. */
LBM_API lbm_status lbm_export_table(lbm_handle* h, int32_t* nei_loc);

/* Chooses ordering x block size x pull-table form by timing `trial_steps`
 * steps of each candidate on this geometry; the state is restored afterwards.
 * Writes the chosen ordering / block size and their measured MLUPS (the
 * table form: lbm_table_info). */
LBM_API lbm_status lbm_autotune(lbm_handle* h, int trial_steps, int* ordering_out, int* block_out,
                        double* mlups_out);

/* Kernel timing of the last lbm_step call (CUDA events on the handle's stream). */
LBM_API lbm_status lbm_last_step_ms(lbm_handle* h, double* ms);

/* Memory facts: bytes of device memory the handle holds and the algorithmic
 * bytes one fluid-node update moves (2*19*s populations + the pull-table
 * bytes of lbm_table_info). */
LBM_API lbm_status lbm_memory(lbm_handle* h, size_t* device_bytes, double* bytes_per_lu);

/* Device memory of every solver (single-phase, colour-gradient, solute, node
 * pool) comes from the device's default CUDA memory pool, and what a
 * destroyed solver frees stays mapped in the process for the next solver
 * (creating one then costs no new mappings).  This returns that cached memory
 * to the driver, for every device the library allocated on; it waits for
 * those devices to be idle. */
LBM_API lbm_status lbm_release_cached_memory(void);

/* Form of the pull table the step kernel reads (the reference's nei_loc,
 * SP3:1099-1151, as a pull table).  compact = 0 (default): the int32 table.
 * compact = 1: per aligned group of 32 nodes and direction one int32 base
 * and per node a 16-bit offset from it, 18*2 + 18*4/32 bytes per node
 * instead of 18*4; groups whose sources spread wider than the offsets reach
 * read the int32 table.  The two give identical results; the compact form
 * moves fewer bytes but waits on more dependent loads, and lbm_autotune
 * times both.  The other kernels (reductions, exports, faces) always read
 * the int32 table.  The compact form (18*2.125 bytes per node of device
 * memory) is built when it is first chosen or asked about, not at creation. */
LBM_API lbm_status lbm_set_table_mode(lbm_handle* h, int compact);
/* current mode, table bytes per node the step reads, and the share of
 * (group, direction) pairs that fall back to the int32 table (asking for
 * the share builds the compact form if it was not built yet) */
LBM_API lbm_status lbm_table_info(lbm_handle* h, int* compact, double* table_bytes_per_node,
                                  double* wide_fraction);

/* ----------------------------------------------- reference output formats */

/* ASCII VTK STRUCTURED_POINTS files of the reference, same header lines and
 * number formatting: LBM_Geometry.vtk (SP3:3205-3247, 0 pore / 1 solid),
 * LBM_velocity_Vector_<n>.vtk (SP3:3286-3377), LBM_Density_<n>.vtk
 * (SP3:3379-3466).  The caller chooses the path. */
LBM_API lbm_status lbm_write_vtk_geometry(const uint8_t* mask, int nx, int ny, int nz, const char* path);
LBM_API lbm_status lbm_write_vtk_velocity(lbm_handle* h, const char* path);
LBM_API lbm_status lbm_write_vtk_density(lbm_handle* h, const char* path);

/* <prefix>LBM_checkpoint_{velocity,rho,f}_<m>.0.bin_input: raw doubles in the
 * reference layout including row 0 (Backup SP3:3469-3516); reading restores
 * the state like Backup_init (SP3:3652-3767). */
LBM_API lbm_status lbm_write_checkpoint(lbm_handle* h, const char* prefix, long long m);
LBM_API lbm_status lbm_read_checkpoint(lbm_handle* h, const char* prefix, long long m);

/* --------------------------------------- colour-gradient two-phase solver */

/* Physics of the colour-gradient model (the INPUT_CG_SPARSE fields of
 * CG3:386-470 that a fully periodic run uses). */
typedef struct lbm_cg_params {
  double nu_l, nu_g;       /* viscosity of component r (psi = 1) and b (psi = -1) */
  double psi_solid;        /* wall colour = cos(contact angle) (ContactAngle_parameter) */
  double cap_a;            /* surface-tension parameter CapA */
  double gx, gy, gz;       /* body force */
  int body_force_phase;    /* 1: only psi >= flux_psi driven, -1: only psi <= -flux_psi, 0: both */
  double flux_psi;         /* rel_perm_psi: phase threshold of forcing and fluxes */
  double flux_umax;        /* rel_perm_psi2: fluxes count nodes with |u| below this */
  int precision;           /* LBM_PREC_F64 (bit-exact) or LBM_PREC_F32 */
  int device;
  int perdir;              /* PerDir 1..3: direction of the permeability change and of sd_l/sd_g */
} lbm_cg_params;

/* Comput_Perm (CG3:5116-5284) and Comput_Saturation (CG3:5286-5370). */
typedef struct lbm_cg_diag {
  long long step;
  double saturation;       /* share of pore nodes with psi >= 0 */
  double q_l[3], q_g[3];   /* phase fluxes (sum of u per phase) */
  double perm_l[3], perm_g[3];
  double perm_rel_change;  /* liquid permeability along perdir, relative change */
  double u_ave;            /* |Q_l + Q_g| / (V * porosity) */
  double capillary;        /* u_ave * nu_l / cap_a */
  double mass;             /* sum rho */
  /* Error (CG3:4683-4750) over all nodes, against u one step earlier */
  double u_max;            /* max |u| */
  double u_rel_change;     /* ||u - u_prev|| / (||u|| + 1e-30) */
  double u_mean_speed;     /* sum |u| / (nx ny nz) */
  /* Comput_Saturation's position sums (CG3:5300-5345): sum of psi * (coordinate
   * along perdir) over nodes with psi >= 0 (sd_l) and psi < 0 (sd_g) */
  double sd_l, sd_g;
} lbm_cg_diag;

typedef struct lbm_cg_handle lbm_cg_handle;

/* mask [nz][ny][nx] (0 = pore), psi [nz][ny][nx] initial phase per cell (the
 * reference's phase file; read as float, CG3:2144-2150). */
LBM_API lbm_status lbm_cg_create(const lbm_cg_params* p, const uint8_t* mask, const double* psi, int nx, int ny,
                                 int nz, lbm_cg_handle** out);
/* As lbm_cg_create with pressure/velocity faces: boundary_pressure
 * (CG3:4221-4682) and boundary_velocity (CG3:4026-4220) with the rules,
 * face lists and quirks of the single-phase solver (the two programs share
 * these functions), acting on the post-streaming populations of the face
 * nodes between collision and the macro step.  in_bc adds the pressure-
 * gradient term |p_+ - p_-| c_s^2 / n_axis to the permeabilities' divisor
 * (Comput_Perm, CG3:5137-5149).  bc may be null (fully periodic).  Replaces
 * the reference's boundary step in its main loop (CG3:868-876). */
LBM_API lbm_status lbm_cg_create_bc(const lbm_cg_params* p, const lbm_boundary* bc, const uint8_t* mask,
                                    const double* psi, int nx, int ny, int nz, lbm_cg_handle** out);
/* Face densities p_xp..p_zn and normal velocities v_xp..v_zn from now on,
 * and whether the face rules run at the steps from now on (the reference
 * runs them only from stab_time when the stabiliser is on, CG3:868).  A
 * change between steps acts on the step just run, as pressure_bodyforce_change
 * and pressure_capillary change p_* between collision and boundary_pressure
 * (CG3:851-871). */
LBM_API lbm_status lbm_cg_set_faces(lbm_cg_handle* h, const double rho[6], const double vel[6], int active);
/* collision (CG3:2546-3290) + comput_macro_variables (CG3:3316-3370), n times */
LBM_API lbm_status lbm_cg_step(lbm_cg_handle* h, int nsteps);
LBM_API lbm_status lbm_cg_reduce(lbm_cg_handle* h, lbm_cg_diag* out);
/* reference id order, row 0 unused; any pointer may be NULL */
LBM_API lbm_status lbm_cg_get_fields(lbm_cg_handle* h, double* rho, double* u, double* psi, double* rho_r,
                                     double* rho_b);
/* post-streaming f in the CG velocity order, [(count+1)*19] */
LBM_API lbm_status lbm_cg_get_populations(lbm_cg_handle* h, double* f);
LBM_API lbm_status lbm_cg_info(lbm_cg_handle* h, int* count, double* porosity, long long* step,
                               double* last_step_ms);
LBM_API void lbm_cg_destroy(lbm_cg_handle* h);

/* Parameter changes between steps (the reference's gxs / CapA updates).
 * timing LBM_CG_FORCE_BEFORE_MACRO: the new force also enters the macro step
 * of the last step taken (pressure_bodyforce_change, CG3:1252-1370, runs
 * between collision and comput_macro_variables); LBM_CG_FORCE_BEFORE_COLLISION:
 * the last step's macro keeps the old force and the next collision uses the
 * new one (the stabiliser's switch at stab_time, CG3:851-852). */
#define LBM_CG_FORCE_BEFORE_MACRO 0
#define LBM_CG_FORCE_BEFORE_COLLISION 1
LBM_API lbm_status lbm_cg_set_body_force(lbm_cg_handle* h, double gx, double gy, double gz, int timing);
/* rel_perm_ift's surface-tension change (CG3:892-893) */
LBM_API lbm_status lbm_cg_set_cap_a(lbm_cg_handle* h, double cap_a);
/* The initial velocity of init (inivx, inivy, inivz, CG3:2357-2400): every
 * node starts from feq(1, u0) of CG3's feq and the first collision takes
 * rho = 1, u = u0.  Only before the first step (LBM_ERR_STATE otherwise). */
LBM_API lbm_status lbm_cg_set_initial_velocity(lbm_cg_handle* h, double ux, double uy, double uz);
/* Comput_Perm / Comput_Saturation window (CG3:5156-5227, 5307-5361):
 * window = per_xn, per_xp, per_yn, per_yp, per_zn, per_zp; the fluxes and the
 * saturation count are divided by its volume, and the porosity (lbm_cg_info,
 * u_ave, capillary number, saturation) becomes the window's pore fraction
 * (CG3:1835-1851).  restrict_nodes = 1 also limits
 * the sums to the nodes inside it (the reference does so when one of
 * par_per_x/y/z equals 1).  All -1 = whole box. */
LBM_API lbm_status lbm_cg_set_window(lbm_cg_handle* h, const int window[6], int restrict_nodes);
/* Phase faces (in_psi_BC = 1, CG3:3386-3700): after every macro step the
 * fluid nodes of each enabled face of the box are set, walking the faces x-,
 * x+, y-, y+, z-, z+ and each face's node list in the reference's order
 * (x faces: z outer, y inner; y faces: z outer, x inner; z faces: y outer,
 * x inner):  1 = the initial phase psi0;  2 = the phase of the node's +x
 * neighbour (periodic; y and z faces copy along x too), except that a node
 * whose +x neighbour is solid resets every node of its face to psi0 before
 * the walk goes on;  3 = +1 when draw % 10000 / 10000 < ini_Sat, else -1,
 * the draws of lbm_cg_set_random numbered from 0 in walk order at every macro
 * step (the reference reseeds from the clock every macro step, CG3:3321, so
 * its pattern is the same for all steps within a second of wall time; here
 * it is the same for every step).  rho_r = (psi + 1)/2, rho_b = 1 - rho_r.
 * faces in INPUT order xp, xn, yp, yn, zp, zn; 0 = off. */
LBM_API lbm_status lbm_cg_set_phase_faces(lbm_cg_handle* h, const int faces[6]);
/* ini_Sat and the seed of the random phase faces (face flag 3) set by the
 * next lbm_cg_set_phase_faces.  Draw k of a seed is the splitmix64 output of
 * seed + (k + 1) * 0x9E3779B97F4A7C15 shifted right by 33 bits (a 31-bit
 * integer, in place of the reference's rand()).  No counterpart in the
 * reference, which seeds from the clock. */
LBM_API lbm_status lbm_cg_set_random(lbm_cg_handle* h, double ini_sat, unsigned long long seed);
/* Mixture injection (mix_psi_thickness > 0 with a phase face at x-): the
 * nodes with x <= x_last relax towards equilibrium moments without the
 * surface-tension terms (CG3:2854-2867); x_last < 0 turns it off. */
LBM_API lbm_status lbm_cg_set_zero_sigma(lbm_cg_handle* h, int x_last);
/* Initial phase of the mixture injection (psi_mixture_ini, CG3:6151-6350) for
 * a [nz][ny][nx] mask: in the plane x = thickness, up to portion x its pore
 * count of pore cells next to a solid (then next to a solid or a marked cell)
 * are marked wetting, in square rings around the plane's centre; cells with
 * x <= thickness whose column's cell in that plane is an unmarked pore get
 * psi = -1, all others +1.  psi_out[nz][ny][nx].  The reference reads outside
 * the plane when ny != nz; here such cells count as not pore. */
LBM_API lbm_status lbm_cg_mixture_phase(const uint8_t* mask, int nx, int ny, int nz, int thickness, double portion,
                                        double* psi_out);
/* Restores a state like Backup_init (CG3:5438-5690): f [(count+1)*19] in the
 * CG velocity order, psi, rho_r, rho_b [(count+1)], reference id order (row 0
 * ignored).  The next step takes psi / rho_r / rho_b as given and rho, u from f. */
LBM_API lbm_status lbm_cg_set_state(lbm_cg_handle* h, const double* f, const double* psi, const double* rho_r,
                                    const double* rho_b);

/* INPUT file of the colour-gradient program (CG3:372-474, field order and
 * types kept; nx, ny, nz as written in the file = NX+1, ...). */
typedef struct lbm_cg_input {
  char geometry_file[256];
  char phase_file[256];
  int nx, ny, nz;
  int n_max;
  double reso;
  int in_bc;
  int in_psi_bc;
  double gx, gy, gz;
  int pre_xp; double p_xp; int pre_xn; double p_xn;
  int pre_yp; double p_yp; int pre_yn; double p_yn;
  int pre_zp; double p_zp; int pre_zn; double p_zn;
  int vel_xp; double v_xp; int vel_xn; double v_xn;
  int vel_yp; double v_yp; int vel_yn; double v_yn;
  int vel_zp; double v_zp; int vel_zn; double v_zn;
  int psi_xp, psi_xn, psi_yp, psi_yn, psi_zp, psi_zn;
  double nu_l, nu_g;
  double contact_angle;          /* ContactAngle_parameter = psi_solid */
  double cap_a;
  double inivx, inivy, inivz;
  double permeability;           /* single-phase permeability (mD) for relative values */
  int wr_per, perdir, fre_re, out_mode, fre_ve, fre_de, fre_psi;
  int lattice_v; double dx_input, dt_input;
  char output_path[256];
  int sub_bc;
  int stab, stab_time;
  double ini_sat;
  int ini_buf;
  double rel_perm_psi, rel_perm_psi2;
  int par_per_x, par_per_y, par_per_z;
  int per_xp, per_xn, per_yp, per_yn, per_zp, per_zn;
  int fre_backup, mode_backup_ini;
  int decbin;
  int pressure_change, pre_chan_pb;
  int pre_chan[5];
  double pre_chan_pn[5], pre_chan_pp[5], pre_chan_f[5];
  int bodyforce_apply;
  int pressure_change2, pre_chan_pb2, interval_pre;
  double pre_chan_pns, pre_chan_pps, pre_chan_fs;
  int chan_no, sat_cri;
  double sat_cri_d;
  int least_square, num_least_square;
  int rel_perm_id_dir, rel_perm_chan_num;
  int rel_perm_ift; double vary_ift;
  int input_dynamic, update_fre;
  int mix_psi_thickness; double protion_w; int zero_sigma_thickness;
} lbm_cg_input;

LBM_API lbm_status lbm_read_cg_input(const char* path, lbm_cg_input* out);
/* input_update (CG3:5765-5925, every update_fre steps when input_dynamic > 0,
 * after the step's collision and ramps, CG3:859-861): the handle-side values
 * of a re-read INPUT file, that is the wall colour (contact_angle), CapA, the
 * flux thresholds (rel_perm_psi, rel_perm_psi2) from the next collision on,
 * and the body force gx, gy, gz from this step's macro step on
 * (LBM_CG_FORCE_BEFORE_MACRO).  n_max, the output intervals and the
 * single-phase permeability are the caller's (the lbm_cg driver re-reads the
 * file with lbm_read_cg_input and takes those too). */
LBM_API lbm_status lbm_cg_input_update(lbm_cg_handle* h, const lbm_cg_input* in);
/* Phase file (CG3:2130-2150): nx*ny*nz whitespace-separated numbers, x
 * fastest, each read as float; out [nz][ny][nx]. */
LBM_API lbm_status lbm_read_phase(const char* path, int nx, int ny, int nz, double* out);
/* Reads the INPUT file, the geometry and the phase file and creates the
 * solver with the file's physics: psi_solid = ContactAngle_parameter, the
 * force off until stab_time when the stabiliser is on, the flux thresholds
 * rel_perm_psi / rel_perm_psi2, PerDir, the permeability window and the
 * pressure/velocity faces (Sub_BC, in_BC; their rules off until stab_time
 * when the stabiliser is on), the phase faces 1-3, the mixture injection
 * (mix_psi_thickness, protion_w, zero_sigma_thickness) and the random initial
 * phase (ini_Sat >= 0, with the window buffer ini_buf).  The reference draws
 * its random numbers from the C library seeded with the clock (CG3:2232,
 * 3321); here they come from the seeded generator of lbm_cg_set_random with
 * seed 0 (lbm_cg_create_from_input_seeded takes the seed).  A non-zero
 * initial velocity is applied (lbm_cg_set_initial_velocity); the imbibition /
 * drainage control turns the phase faces on as the reference's init does,
 * the control itself and the re-reads of input_dynamic are the caller's
 * (lbm_cg runs both).  A self-defined lattice velocity, and settings the
 * reference would divide by zero on (update_fre, freRe, frePsi = 0), are
 * rejected with LBM_ERR_ARG naming the field. */
LBM_API lbm_status lbm_cg_create_from_input(const char* input_path, int precision, lbm_cg_handle** out,
                                            lbm_cg_input* parsed_out);
/* lbm_cg_create_from_input with the seed of the random initial phase and
 * the random phase faces (no counterpart in the reference, which seeds from
 * the clock). */
LBM_API lbm_status lbm_cg_create_from_input_seeded(const char* input_path, int precision, unsigned long long seed,
                                                   lbm_cg_handle** out, lbm_cg_input* parsed_out);

/* Output writers of the colour-gradient program: velocity and density VTK
 * (output_velocity CG3:4840-4931, output_density CG3:4933-5020; the
 * single-phase formats), the phase VTK (output_psi CG3:5022-5114: title lines
 * given by the caller, values at 2 significant digits, 0 on solids) and the
 * checkpoint <prefix>LBM_checkpoint_{velocity,rho,psi,f,rhor,rhob}_<m>.0.bin_input
 * (Backup CG3:5693-5745; Backup_init CG3:5438-5690 reads it back). */
LBM_API lbm_status lbm_cg_write_vtk_velocity(lbm_cg_handle* h, const char* path);
LBM_API lbm_status lbm_cg_write_vtk_density(lbm_cg_handle* h, const char* path);
LBM_API lbm_status lbm_cg_write_vtk_psi(lbm_cg_handle* h, const char* path, const char* version_suffix,
                                        const char* title);
LBM_API lbm_status lbm_cg_write_checkpoint(lbm_cg_handle* h, const char* prefix, long long m);
LBM_API lbm_status lbm_cg_read_checkpoint(lbm_cg_handle* h, const char* prefix, long long m);

/* --------------------------------------------- D3Q7 solute (passive scalar) */

typedef struct lbm_st7_params {
  double diffusivity;  /* niu_s: tau_s = 3 niu_s + 1/2 (ST7:1262) */
  int precision;       /* LBM_PREC_F64 (reference arithmetic) or LBM_PREC_F32 */
  int device;
} lbm_st7_params;

typedef struct lbm_st7_handle lbm_st7_handle;

/* u_nodes: advecting velocity per fluid node, [(count+1)*3] in the library's
 * reference id order (SP3 compaction, the order lbm_get_fields returns);
 * c0: initial concentration per cell [nz][ny][nx] (the reference's initial
 * concentration file, ST7:1269). */
LBM_API lbm_status lbm_st7_create(const lbm_st7_params* p, const uint8_t* mask, int nx, int ny, int nz,
                                  const double* u_nodes, const double* c0, lbm_st7_handle** out);
/* Same, taking the velocity of a single-phase solve's current state (the
 * flow -> solute coupling of SP:5093-5120 / ST7:3640-3667 without files). */
LBM_API lbm_status lbm_st7_create_from_flow(const lbm_st7_params* p, lbm_handle* flow, const double* c0,
                                            lbm_st7_handle** out);
/* The D3Q19 solute program (ST19 = Single_Phase_3D/
 * Solute_Transport_MPI_Software_Spars.cpp; collision ST19:1346-1640): BGK on
 * the 19 flow directions towards w_q C (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u.u),
 * C = sum of the 19 g in the program's direction order (ST19:121-127, the
 * colour-gradient order).  Same arguments and handle as lbm_st7_create; the
 * lbm_st7_* calls below work on it, with 19 columns for populations. */
LBM_API lbm_status lbm_st19_create(const lbm_st7_params* p, const uint8_t* mask, int nx, int ny, int nz,
                                   const double* u_nodes, const double* c0, lbm_st7_handle** out);
LBM_API lbm_status lbm_st19_create_from_flow(const lbm_st7_params* p, lbm_handle* flow, const double* c0,
                                             lbm_st7_handle** out);
/* Directions of a solute handle: 7 (lbm_st7_create*) or 19 (lbm_st19_create*);
 * 0 for a null handle. */
LBM_API int lbm_st7_directions(lbm_st7_handle* h);
/* collision + streaming + C = sum g (ST7:1345-1633), n times */
/* Self-defined lattice velocity (lattice_v with dx, dt of the INPUT file,
 * ST7:1259-1274, the D3Q19 program the same): tau_s = niu_s / (c_s^2 dt) + 1/2
 * with c_s^2 = (dx/dt)^2 / 3, and the D3Q19 equilibrium's e.u and u.u terms
 * divided by c2 = (dx/dt)^2 and c4 = c2^2 as the program divides them.  The
 * default lattice is dx = dt = 1. */
LBM_API lbm_status lbm_st7_set_lattice(lbm_st7_handle* h, double dx, double dt);
LBM_API lbm_status lbm_st7_step(lbm_st7_handle* h, int nsteps);
/* C per fluid node [(count+1)], reference id order, row 0 zero */
LBM_API lbm_status lbm_st7_get_concentration(lbm_st7_handle* h, double* c);
LBM_API lbm_status lbm_st7_info(lbm_st7_handle* h, int* count, long long* step, double* last_step_ms);
/* g as the next step reads it (the reference's fg after comput_macro_variables,
 * ST7:1619-1633): [(count+1)*7] in reference id order, column 0 and row 0 zero;
 * for a D3Q19 handle [(count+1)*19] in the program's direction order */
LBM_API lbm_status lbm_st7_get_populations(lbm_st7_handle* h, double* g);
/* Restores g [(count+1)*7] ([(count+1)*19] for D3Q19) and C [(count+1)] like
 * Backup_init (ST7:3716-3802); the next step takes C as given */
LBM_API lbm_status lbm_st7_set_state(lbm_st7_handle* h, const double* g, const double* c);

/* INPUT file of the solute program (ST7:219-280, field order and types kept;
 * nx, ny, nz as written in the file). */
typedef struct lbm_st7_input {
  char geometry_file[256];
  char conc_file[256];        /* initial concentration, x fastest, read as float */
  int nx, ny, nz;
  int n_max;
  double reso;
  int in_bc;
  double buoyancy, ref_psi;   /* ref_psi: value written on solid cells */
  double gravity;
  double gx, gy, gz;
  int pre_xp; double p_xp; int pre_xn; double p_xn;
  int pre_yp; double p_yp; int pre_yn; double p_yn;
  int pre_zp; double p_zp; int pre_zn; double p_zn;
  int vel_xp; double v_xp; int vel_xn; double v_xn;
  int vel_yp; double v_yp; int vel_yn; double v_yn;
  int vel_zp; double v_zp; int vel_zn; double v_zn;
  int sol_c_xp; double c_xp; int sol_c_xn; double c_xn;
  int sol_c_yp; double c_yp; int sol_c_yn; double c_yn;
  int sol_c_zp; double c_zp; int sol_c_zn; double c_zn;
  int sol_zf_xp; double zf_xp; int sol_zf_xn; double zf_xn;
  int sol_zf_yp; double zf_yp; int sol_zf_yn; double zf_yn;
  int sol_zf_zp; double zf_zp; int sol_zf_zn; double zf_zn;
  double nu;                  /* flow viscosity (for the Reynolds number) */
  double nu_s;                /* solute diffusivity */
  double inivx, inivy, inivz;
  int wr_per, perdir, fre_re, out_mode, fre_ve, fre_de, fre_psi;
  int sub_dis, fre_dis;
  int lattice_v; double dx_input, dt_input;
  char output_path[256];
  int sub_bc, sub_bc_psi, ini_psi;
  int par_per_x, par_per_y, par_per_z;
  int per_xp, per_xn, per_yp, per_yn, per_zp, per_zn;
  int fre_backup, mode_backup_ini;
  int sol_ini_n;              /* step tag of the Velocity_for_solute files read */
  int decbin;
} lbm_st7_input;

LBM_API lbm_status lbm_read_st7_input(const char* path, lbm_st7_input* out);

/* x-slab decomposition of the slab programs (ST7:951-975): rank r holds the
 * x-planes [first_x[r], first_x[r+1]), first_x [nranks+1].  The per-rank
 * Velocity_for_solute and checkpoint files of an N-rank run follow it. */
LBM_API lbm_status lbm_slab_partition(const uint8_t* mask, int nx, int ny, int nz, int nranks, int* first_x);
LBM_API void lbm_st7_destroy(lbm_st7_handle* h);

/* Velocity_for_solute_<n>.<rank>.bin (SP:5093-5120): Count*3 raw doubles in
 * the slab solver's compaction order at one rank (i outer, j, k inner).
 * Write from a single-phase solve's current velocity; read into the
 * library's id order ([(count+1)*3], row 0 zero). */
LBM_API lbm_status lbm_write_velocity_for_solute(lbm_handle* flow, const char* path);
LBM_API lbm_status lbm_read_velocity_for_solute(const char* path, const uint8_t* mask, int nx, int ny, int nz,
                                                double* u_nodes);

/* The same file in either record order.  LBM_SOLUTE_ORDER_SLAB is the one
 * above (written by SP:5093-5120, read by the solute programs,
 * Backup_input_v, Solute_Transport_MPI_Software_Spars.cpp:3649-3690); LBM_SOLUTE_ORDER_XFAST
 * is what the 3-D partition program writes at one rank
 * (output_velocity_for_solute, SP3:3769-3797): pore cells with x fastest. */
typedef enum { LBM_SOLUTE_ORDER_SLAB = 0, LBM_SOLUTE_ORDER_XFAST = 1 } lbm_solute_order;
LBM_API lbm_status lbm_write_velocity_for_solute_ordered(lbm_handle* flow, const char* path, int order);
LBM_API lbm_status lbm_read_velocity_for_solute_ordered(const char* path, const uint8_t* mask, int nx, int ny,
                                                        int nz, int order, double* u_nodes);

/* ------------------------------------------ many independent solves (pool) */

/* One single-phase permeability solve: geometry and physics (fully periodic,
 * rest initial state, whole-box permeability window). */
typedef struct lbm_instance {
  const uint8_t* mask;  /* [nz][ny][nx], 0 = pore; copied by the library */
  int nx, ny, nz;
  double nu;            /* viscosity; tau = 3 nu + 1/2 */
  double gx, gy, gz;    /* body force (acceleration) */
} lbm_instance;

/* Outcome of one solve run to the reference's stop test
 * |(u_ave_prev - u_ave)/u_ave_prev| < tol checked every check_every steps
 * (SP:812-816), u_ave and permeability from Comput_Perm (SP3:3611-3638). */
typedef struct lbm_solve_result {
  long long steps;   /* steps run */
  int status;        /* LBM_OK converged, LBM_ERR_NOT_CONVERGED cap, LBM_ERR_NAN */
  int count;         /* fluid nodes */
  double perm[3];    /* Q_d / V * nu / g_d */
  double u_ave;      /* |Q| / (V * porosity) */
  double porosity;
  double mass;       /* sum rho */
} lbm_solve_result;

typedef struct lbm_batch lbm_batch;

/* Packs n solves of arbitrary sizes into one node pool (each instance a
 * contiguous tile-aligned node range, its pull table pointing only into its
 * own range) stepped by one persistent kernel per step inside CUDA graphs.
 * precision: LBM_PREC_F32 or LBM_PREC_F16; ordering: node order inside each
 * instance; block: 128/256/512 (0 = 256).  Replaces running the reference
 * binary once per subsample. */
LBM_API lbm_status lbm_batch_create(int n, const lbm_instance* inst, int precision, int ordering, int block,
                                    int device, lbm_batch** out);
/* Runs every instance to convergence (or max_steps); instances that converge
 * stop stepping while the others continue.  results[n] may be NULL. */
LBM_API lbm_status lbm_batch_run(lbm_batch* b, double tol, int check_every, long long max_steps,
                                 lbm_solve_result* results);
/* Puts every instance back to its initial state (rest, rho = 1). */
LBM_API lbm_status lbm_batch_reset(lbm_batch* b);
/* rho[(count_i+1)], u[(count_i+1)*3] of instance i in its reference id order. */
LBM_API lbm_status lbm_batch_get_fields(lbm_batch* b, int i, double* rho, double* u);
/* Picks the step block size and the node ordering by timing trial_steps
 * steps of the whole batch for each candidate; resets the batch. */
LBM_API lbm_status lbm_batch_autotune(lbm_batch* b, int trial_steps, int* ordering_out, int* block_out,
                                      double* mlups_out);
/* total fluid nodes, device time of the last lbm_batch_run (ms), steps summed
 * over instances in that run. */
LBM_API lbm_status lbm_batch_info(lbm_batch* b, long long* total_nodes, double* last_run_ms,
                                  long long* node_steps);
/* No counterpart in the reference (it solves one domain per program run).
 * Per-chain record of the last lbm_batch_run: rows of three doubles --
 * fluid nodes of the instances stepping when the chain started, steps in the
 * chain, device time of the chain in ms (list, steps and per-instance stop
 * test).  Writes min(rows, max_rows) rows; *n_rows = rows recorded. */
LBM_API lbm_status lbm_batch_trace(lbm_batch* b, double* out, int max_rows, int* n_rows);
LBM_API void lbm_batch_destroy(lbm_batch* b);

/* ---------------------------------------- continuous-batching solve server */

typedef struct lbm_server_config {
  long long capacity_nodes;  /* HBM budget of the node pool, in fluid nodes */
  int max_active;            /* slots: solves resident at once */
  int precision;             /* LBM_PREC_F32 or LBM_PREC_F16 */
  int ordering;              /* node order inside each solve */
  int block;                 /* step block size (0 = 256) */
  double tol;                /* stop test tolerance */
  int check_every;           /* steps per device chain between admissions */
  long long max_steps;       /* per-solve step cap */
  int device;
  long long target_active_nodes; /* admit while resident nodes are below this
                                    (0 = no limit but memory): enough nodes to
                                    keep HBM busy, no more, so each resident
                                    solve gets a large share of the device */
  int policy;                /* admission order: LBM_SERVE_FIFO (arrival) or
                                LBM_SERVE_SHORTEST_FIRST (least estimated
                                work first: cells x nx^2; a stream of small
                                requests can hold a large one back) */
} lbm_server_config;
#define LBM_SERVE_FIFO 0
#define LBM_SERVE_SHORTEST_FIRST 1

typedef struct lbm_server_result {
  long long request_id;
  lbm_solve_result result;
  double t_submit, t_admit, t_done;  /* seconds on the server's steady clock */
} lbm_server_result;

typedef struct lbm_server lbm_server;

LBM_API void lbm_server_config_default(lbm_server_config* c);
LBM_API lbm_status lbm_server_create(const lbm_server_config* c, lbm_server** out);
/* Queues a solve (the mask is copied).  Requests larger than the whole pool
 * are rejected with LBM_ERR_ARG. */
LBM_API lbm_status lbm_server_submit(lbm_server* s, const lbm_instance* req, long long* request_id);
/* One round: the resident solves advance check_every steps on the device
 * while the host prepares queued requests; finished solves are retired and
 * their nodes freed; queued requests are admitted (first fit, in the
 * policy's order with skip-ahead) as slots and pool memory allow. */
LBM_API lbm_status lbm_server_pump(lbm_server* s, int* n_active, int* n_queued);
/* Moves up to max finished results into out; *n_out = number written. */
LBM_API lbm_status lbm_server_poll(lbm_server* s, lbm_server_result* out, int max, int* n_out);
/* Seconds on the server's clock (the same clock as the result stamps). */
LBM_API double lbm_server_now(lbm_server* s);
LBM_API void lbm_server_destroy(lbm_server* s);

/* No counterpart in the reference: an addition for callers that cannot
 * allocate device memory (a host framework that owns every allocation and
 * hands libraries its own arena, code in a region where cudaMalloc is not
 * allowed or would synchronise the device).  It computes the same eight
 * diagnostic sums as lbm_reduce -- sum |u - u_prev|^2, sum |u|^2, sum |u|,
 * max |u|^2 (all without node skip_node, the reference's last node), Q_x,
 * Q_y, Q_z, sum rho -- from caller-owned device arrays and writes them to
 * result_dev[8], allocating nothing:
 *   f_dev       post-streaming populations, FP64, f_q of node p at
 *               f_dev[q*stride + p] (19 rows)
 *   u_prev_dev  velocity one step earlier, [3][stride], or NULL (zero change)
 *   n, stride   nodes and row stride (stride >= n)
 *   stream      a cudaStream_t, or NULL for the default stream; the call is
 *               asynchronous on it
 * Its scratch (one row of partial sums per 2048-node tile) is a static
 * device array of 512 KiB that every GPU loading the library holds until the
 * process exits, so n is limited to 16,777,216 nodes; larger n is rejected
 * with LBM_ERR_ARG.  Every call looks up the array's device address on the
 * current device (cudaGetSymbolAddress allocates nothing), so the address
 * stays valid after a cudaDeviceReset; the first call on a device also loads
 * the library's kernels there, so make that first call before any stream
 * capture.  All calls share the one array and every call
 * overwrites it: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
LBM_API lbm_status lbm_reduce_noalloc(const double* f_dev, const double* u_prev_dev, int n, int stride,
                                      int skip_node, double gx, double gy, double gz, double* result_dev,
                                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
