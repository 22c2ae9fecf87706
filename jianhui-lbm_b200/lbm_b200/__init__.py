"""Python front-end of liblbm.so (the B200 sparse D3Q19 lattice Boltzmann library).

This module only binds the C ABI declared in include/lbm.h with ctypes; all
compute runs in the native library.  There is no fallback: if liblbm.so is
missing or has no kernel image for the GPU, the import or the first call
fails with an error.

The names mirror the reference's solver surface (Single_Phase_3D/
SINGLE_PHASE_MPI_Software_Spars_3DPartition.cpp): ``step`` is its time loop
body (collision + comput_macro_variables), ``reduce`` is Error +
Comput_Perm, ``fields``/``populations`` return the reference's rho/u/f arrays
in its own id order and layout.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbm.so")

PREC_F64, PREC_F32, PREC_F16, PREC_F64_FAST = 0, 1, 2, 3
ORDER_REFERENCE, ORDER_MORTON, ORDER_HILBERT, ORDER_BRICK, ORDER_AUTO = 0, 1, 2, 3, -1

PRECISIONS = {"f64": PREC_F64, "f32": PREC_F32, "f16": PREC_F16, "f64fast": PREC_F64_FAST}
ORDERINGS = {"reference": ORDER_REFERENCE, "morton": ORDER_MORTON, "hilbert": ORDER_HILBERT,
             "brick": ORDER_BRICK, "auto": ORDER_AUTO}

STATUS = {
    0: "LBM_OK", -1: "LBM_ERR_ARG", -2: "LBM_ERR_IO", -3: "LBM_ERR_OOM", -4: "LBM_ERR_CUDA",
    -5: "LBM_ERR_NAN", -6: "LBM_ERR_NOT_CONVERGED", -7: "LBM_ERR_FORMAT", -8: "LBM_ERR_STATE",
    -9: "LBM_ERR_OVERSPEED", -10: "LBM_ERR_NO_DEVICE",
}


class LbmError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Boundary(C.Structure):
    """lbm_boundary: pressure/velocity faces, INPUT.dat order xp, xn, yp, yn, zp, zn."""
    _fields_ = [
        ("sub_bc", C.c_int), ("in_bc", C.c_int), ("pressure", C.c_int * 6), ("rho", C.c_double * 6),
        ("velocity", C.c_int * 6), ("vel", C.c_double * 6),
    ]

    @classmethod
    def make(cls, sub_bc=0, in_bc=0, pressure=(0,) * 6, rho=(1.0,) * 6, velocity=(0,) * 6, vel=(0.0,) * 6):
        return cls(int(sub_bc), int(in_bc), (C.c_int * 6)(*[int(x) for x in pressure]),
                   (C.c_double * 6)(*[float(x) for x in rho]), (C.c_int * 6)(*[int(x) for x in velocity]),
                   (C.c_double * 6)(*[float(x) for x in vel]))


class Params(C.Structure):
    _fields_ = [
        ("nu", C.c_double), ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
        ("u_init", C.c_double * 3), ("precision", C.c_int), ("ordering", C.c_int),
        ("block_size", C.c_int), ("perdir", C.c_int), ("window", C.c_int * 6),
        ("fp16_scale", C.c_double), ("device", C.c_int), ("bc", Boundary),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("step", C.c_longlong), ("perm", C.c_double * 3), ("perm_rel_change", C.c_double),
        ("u_ave", C.c_double), ("u_max", C.c_double), ("u_rel_change", C.c_double),
        ("u_mean_speed", C.c_double), ("mass", C.c_double), ("porosity", C.c_double),
        ("nan_detected", C.c_int), ("converged", C.c_int),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["perm"] = list(self.perm)
        return d


class Input(C.Structure):
    _fields_ = [
        ("geometry_file", C.c_char * 128), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("n_max", C.c_int), ("reso", C.c_double), ("in_bc", C.c_int),
        ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
        ("pre_xp", C.c_int), ("p_xp", C.c_double), ("pre_xn", C.c_int), ("p_xn", C.c_double),
        ("pre_yp", C.c_int), ("p_yp", C.c_double), ("pre_yn", C.c_int), ("p_yn", C.c_double),
        ("pre_zp", C.c_int), ("p_zp", C.c_double), ("pre_zn", C.c_int), ("p_zn", C.c_double),
        ("vel_xp", C.c_int), ("v_xp", C.c_double), ("vel_xn", C.c_int), ("v_xn", C.c_double),
        ("vel_yp", C.c_int), ("v_yp", C.c_double), ("vel_yn", C.c_int), ("v_yn", C.c_double),
        ("vel_zp", C.c_int), ("v_zp", C.c_double), ("vel_zn", C.c_int), ("v_zn", C.c_double),
        ("in_vis", C.c_double), ("inivx", C.c_double), ("inivy", C.c_double), ("inivz", C.c_double),
        ("wr_per", C.c_int), ("perdir", C.c_int), ("fre_re", C.c_int), ("out_mode", C.c_int),
        ("fre_ve", C.c_int), ("fre_de", C.c_int),
        ("lattice_v", C.c_int), ("dx_input", C.c_double), ("dt_input", C.c_double),
        ("output_path", C.c_char * 128), ("sub_bc", C.c_int), ("loc_perm", C.c_int),
        ("par_per_x", C.c_int), ("par_per_y", C.c_int), ("par_per_z", C.c_int),
        ("per_xp", C.c_int), ("per_xn", C.c_int), ("per_yp", C.c_int), ("per_yn", C.c_int),
        ("per_zp", C.c_int), ("per_zn", C.c_int),
        ("fre_backup", C.c_int), ("mode_backup_ini", C.c_int), ("vel_sol", C.c_int),
        ("gperm", C.c_int), ("n_gperm", C.c_int * 4), ("size_gperm", C.c_int * 4),
        ("c_gperm", (C.c_int * 3) * 4), ("decbin", C.c_int),
        ("nnf_module", C.c_int), ("nnf_m", C.c_double), ("nnf_n", C.c_double),
    ]

    def as_dict(self):
        out = {}
        for k, t in self._fields_:
            v = getattr(self, k)
            if isinstance(v, bytes):
                v = v.decode()
            elif hasattr(v, "__len__"):
                v = [list(x) if hasattr(x, "__len__") else x for x in v]
            out[k] = v
        return out


class Instance(C.Structure):
    _fields_ = [("mask", C.c_void_p), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nu", C.c_double),
                ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double)]


class SolveResult(C.Structure):
    _fields_ = [("steps", C.c_longlong), ("status", C.c_int), ("count", C.c_int), ("perm", C.c_double * 3),
                ("u_ave", C.c_double), ("porosity", C.c_double), ("mass", C.c_double)]

    def as_dict(self):
        return {"steps": self.steps, "status": self.status, "count": self.count, "perm": list(self.perm),
                "u_ave": self.u_ave, "porosity": self.porosity, "mass": self.mass}


class ServerConfig(C.Structure):
    _fields_ = [("capacity_nodes", C.c_longlong), ("max_active", C.c_int), ("precision", C.c_int),
                ("ordering", C.c_int), ("block", C.c_int), ("tol", C.c_double), ("check_every", C.c_int),
                ("max_steps", C.c_longlong), ("device", C.c_int), ("target_active_nodes", C.c_longlong),
                ("policy", C.c_int)]


class ServerResult(C.Structure):
    _fields_ = [("request_id", C.c_longlong), ("result", SolveResult), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double)]


class CGParams(C.Structure):
    _fields_ = [("nu_l", C.c_double), ("nu_g", C.c_double), ("psi_solid", C.c_double), ("cap_a", C.c_double),
                ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double), ("body_force_phase", C.c_int),
                ("flux_psi", C.c_double), ("flux_umax", C.c_double), ("precision", C.c_int), ("device", C.c_int),
                ("perdir", C.c_int)]


class CGInput(C.Structure):
    _fields_ = [
        ("geometry_file", C.c_char * 256), ("phase_file", C.c_char * 256),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("n_max", C.c_int), ("reso", C.c_double),
        ("in_bc", C.c_int), ("in_psi_bc", C.c_int), ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
        ("pre_xp", C.c_int), ("p_xp", C.c_double), ("pre_xn", C.c_int), ("p_xn", C.c_double),
        ("pre_yp", C.c_int), ("p_yp", C.c_double), ("pre_yn", C.c_int), ("p_yn", C.c_double),
        ("pre_zp", C.c_int), ("p_zp", C.c_double), ("pre_zn", C.c_int), ("p_zn", C.c_double),
        ("vel_xp", C.c_int), ("v_xp", C.c_double), ("vel_xn", C.c_int), ("v_xn", C.c_double),
        ("vel_yp", C.c_int), ("v_yp", C.c_double), ("vel_yn", C.c_int), ("v_yn", C.c_double),
        ("vel_zp", C.c_int), ("v_zp", C.c_double), ("vel_zn", C.c_int), ("v_zn", C.c_double),
        ("psi_xp", C.c_int), ("psi_xn", C.c_int), ("psi_yp", C.c_int), ("psi_yn", C.c_int), ("psi_zp", C.c_int),
        ("psi_zn", C.c_int), ("nu_l", C.c_double), ("nu_g", C.c_double), ("contact_angle", C.c_double),
        ("cap_a", C.c_double), ("inivx", C.c_double), ("inivy", C.c_double), ("inivz", C.c_double),
        ("permeability", C.c_double), ("wr_per", C.c_int), ("perdir", C.c_int), ("fre_re", C.c_int),
        ("out_mode", C.c_int), ("fre_ve", C.c_int), ("fre_de", C.c_int), ("fre_psi", C.c_int),
        ("lattice_v", C.c_int), ("dx_input", C.c_double), ("dt_input", C.c_double),
        ("output_path", C.c_char * 256), ("sub_bc", C.c_int), ("stab", C.c_int), ("stab_time", C.c_int),
        ("ini_sat", C.c_double), ("ini_buf", C.c_int), ("rel_perm_psi", C.c_double), ("rel_perm_psi2", C.c_double),
        ("par_per_x", C.c_int), ("par_per_y", C.c_int), ("par_per_z", C.c_int),
        ("per_xp", C.c_int), ("per_xn", C.c_int), ("per_yp", C.c_int), ("per_yn", C.c_int),
        ("per_zp", C.c_int), ("per_zn", C.c_int), ("fre_backup", C.c_int), ("mode_backup_ini", C.c_int),
        ("decbin", C.c_int), ("pressure_change", C.c_int), ("pre_chan_pb", C.c_int), ("pre_chan", C.c_int * 5),
        ("pre_chan_pn", C.c_double * 5), ("pre_chan_pp", C.c_double * 5), ("pre_chan_f", C.c_double * 5),
        ("bodyforce_apply", C.c_int), ("pressure_change2", C.c_int), ("pre_chan_pb2", C.c_int),
        ("interval_pre", C.c_int), ("pre_chan_pns", C.c_double), ("pre_chan_pps", C.c_double),
        ("pre_chan_fs", C.c_double), ("chan_no", C.c_int), ("sat_cri", C.c_int), ("sat_cri_d", C.c_double),
        ("least_square", C.c_int), ("num_least_square", C.c_int), ("rel_perm_id_dir", C.c_int),
        ("rel_perm_chan_num", C.c_int), ("rel_perm_ift", C.c_int), ("vary_ift", C.c_double),
        ("input_dynamic", C.c_int), ("update_fre", C.c_int), ("mix_psi_thickness", C.c_int),
        ("protion_w", C.c_double), ("zero_sigma_thickness", C.c_int),
    ]

    as_dict = Input.as_dict


class ST7Input(C.Structure):
    _fields_ = [
        ("geometry_file", C.c_char * 256), ("conc_file", C.c_char * 256),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("n_max", C.c_int), ("reso", C.c_double),
        ("in_bc", C.c_int), ("buoyancy", C.c_double), ("ref_psi", C.c_double), ("gravity", C.c_double),
        ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
    ] + [item for ax in "xyz" for item in ((f"pre_{ax}p", C.c_int), (f"p_{ax}p", C.c_double),
                                          (f"pre_{ax}n", C.c_int), (f"p_{ax}n", C.c_double))] \
      + [item for ax in "xyz" for item in ((f"vel_{ax}p", C.c_int), (f"v_{ax}p", C.c_double),
                                          (f"vel_{ax}n", C.c_int), (f"v_{ax}n", C.c_double))] \
      + [item for ax in "xyz" for item in ((f"sol_c_{ax}p", C.c_int), (f"c_{ax}p", C.c_double),
                                          (f"sol_c_{ax}n", C.c_int), (f"c_{ax}n", C.c_double))] \
      + [item for ax in "xyz" for item in ((f"sol_zf_{ax}p", C.c_int), (f"zf_{ax}p", C.c_double),
                                          (f"sol_zf_{ax}n", C.c_int), (f"zf_{ax}n", C.c_double))] \
      + [("nu", C.c_double), ("nu_s", C.c_double), ("inivx", C.c_double), ("inivy", C.c_double),
         ("inivz", C.c_double), ("wr_per", C.c_int), ("perdir", C.c_int), ("fre_re", C.c_int),
         ("out_mode", C.c_int), ("fre_ve", C.c_int), ("fre_de", C.c_int), ("fre_psi", C.c_int),
         ("sub_dis", C.c_int), ("fre_dis", C.c_int), ("lattice_v", C.c_int), ("dx_input", C.c_double),
         ("dt_input", C.c_double), ("output_path", C.c_char * 256), ("sub_bc", C.c_int), ("sub_bc_psi", C.c_int),
         ("ini_psi", C.c_int), ("par_per_x", C.c_int), ("par_per_y", C.c_int), ("par_per_z", C.c_int),
         ("per_xp", C.c_int), ("per_xn", C.c_int), ("per_yp", C.c_int), ("per_yn", C.c_int),
         ("per_zp", C.c_int), ("per_zn", C.c_int), ("fre_backup", C.c_int), ("mode_backup_ini", C.c_int),
         ("sol_ini_n", C.c_int), ("decbin", C.c_int)]

    as_dict = Input.as_dict


class CGDiag(C.Structure):
    _fields_ = [("step", C.c_longlong), ("saturation", C.c_double), ("q_l", C.c_double * 3),
                ("q_g", C.c_double * 3), ("perm_l", C.c_double * 3), ("perm_g", C.c_double * 3),
                ("perm_rel_change", C.c_double), ("u_ave", C.c_double), ("capillary", C.c_double),
                ("mass", C.c_double), ("u_max", C.c_double), ("u_rel_change", C.c_double),
                ("u_mean_speed", C.c_double), ("sd_l", C.c_double), ("sd_g", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        for k in ("q_l", "q_g", "perm_l", "perm_g"):
            d[k] = list(d[k])
        return d


_lib = None
_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_U8P = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")

# name -> (argtypes, restype)
_SIGNATURES = {
    "lbm_last_error": ([], C.c_char_p),
    "lbm_status_string": ([C.c_int], C.c_char_p),
    "lbm_abi_version": ([], C.c_int),
    "lbm_params_default": ([C.POINTER(Params)], None),
    "lbm_read_input": ([C.c_char_p, C.POINTER(Input)], C.c_int),
    "lbm_read_mask": ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, _U8P], C.c_int),
    "lbm_create": ([C.POINTER(Params), _U8P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "lbm_create_from_input": ([C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_void_p), C.POINTER(Input)], C.c_int),
    "lbm_destroy": ([C.c_void_p], None),
    "lbm_step": ([C.c_void_p, C.c_int], C.c_int),
    "lbm_reduce": ([C.c_void_p, C.POINTER(Diag)], C.c_int),
    "lbm_run_to_convergence": ([C.c_void_p, C.c_double, C.c_int, C.c_int, C.POINTER(Diag)], C.c_int),
    "lbm_info": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_longlong)], C.c_int),
    "lbm_get_fields": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "lbm_get_populations": ([C.c_void_p, _F64P], C.c_int),
    "lbm_set_state": ([C.c_void_p, _F64P, _F64P, _F64P], C.c_int),
    "lbm_export_compaction": ([C.c_void_p, _I32P], C.c_int),
    "lbm_export_table": ([C.c_void_p, _I32P], C.c_int),
    "lbm_autotune": ([C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
    "lbm_last_step_ms": ([C.c_void_p, C.POINTER(C.c_double)], C.c_int),
    "lbm_memory": ([C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_double)], C.c_int),
    "lbm_set_table_mode": ([C.c_void_p, C.c_int], C.c_int),
    "lbm_set_lattice": ([C.c_void_p, C.c_double, C.c_double], C.c_int),
    "lbm_release_cached_memory": ([], C.c_int),
    "lbm_table_info": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "lbm_reduce_noalloc": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                            C.c_void_p, C.c_void_p], C.c_int),
    "lbm_batch_create": ([C.c_int, C.POINTER(Instance), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
                         C.c_int),
    "lbm_batch_run": ([C.c_void_p, C.c_double, C.c_int, C.c_longlong, C.POINTER(SolveResult)], C.c_int),
    "lbm_batch_reset": ([C.c_void_p], C.c_int),
    "lbm_batch_get_fields": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "lbm_batch_autotune": ([C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)],
                           C.c_int),
    "lbm_batch_info": ([C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_double), C.POINTER(C.c_longlong)], C.c_int),
    "lbm_batch_trace": ([C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "lbm_batch_destroy": ([C.c_void_p], None),
    "lbm_server_config_default": ([C.POINTER(ServerConfig)], None),
    "lbm_server_create": ([C.POINTER(ServerConfig), C.POINTER(C.c_void_p)], C.c_int),
    "lbm_server_submit": ([C.c_void_p, C.POINTER(Instance), C.POINTER(C.c_longlong)], C.c_int),
    "lbm_server_pump": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "lbm_server_poll": ([C.c_void_p, C.POINTER(ServerResult), C.c_int, C.POINTER(C.c_int)], C.c_int),
    "lbm_server_now": ([C.c_void_p], C.c_double),
    "lbm_server_destroy": ([C.c_void_p], None),
    "lbm_cg_create": ([C.POINTER(CGParams), _U8P, _F64P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "lbm_cg_step": ([C.c_void_p, C.c_int], C.c_int),
    "lbm_cg_reduce": ([C.c_void_p, C.POINTER(CGDiag)], C.c_int),
    "lbm_cg_get_fields": ([C.c_void_p] + [C.c_void_p] * 5, C.c_int),
    "lbm_cg_get_populations": ([C.c_void_p, _F64P], C.c_int),
    "lbm_cg_info": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                     C.POINTER(C.c_double)], C.c_int),
    "lbm_cg_destroy": ([C.c_void_p], None),
    "lbm_cg_set_body_force": ([C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int], C.c_int),
    "lbm_cg_set_cap_a": ([C.c_void_p, C.c_double], C.c_int),
    "lbm_cg_input_update": ([C.c_void_p, C.POINTER(CGInput)], C.c_int),
    "lbm_cg_set_initial_velocity": ([C.c_void_p, C.c_double, C.c_double, C.c_double], C.c_int),
    "lbm_cg_create_bc": ([C.POINTER(CGParams), C.POINTER(Boundary), _U8P, _F64P, C.c_int, C.c_int, C.c_int,
                          C.POINTER(C.c_void_p)], C.c_int),
    "lbm_cg_set_faces": ([C.c_void_p, _F64P, _F64P, C.c_int], C.c_int),
    "lbm_cg_set_window": ([C.c_void_p, _I32P, C.c_int], C.c_int),
    "lbm_cg_set_state": ([C.c_void_p, _F64P, _F64P, _F64P, _F64P], C.c_int),
    "lbm_cg_set_phase_faces": ([C.c_void_p, _I32P], C.c_int),
    "lbm_cg_set_zero_sigma": ([C.c_void_p, C.c_int], C.c_int),
    "lbm_cg_set_random": ([C.c_void_p, C.c_double, C.c_ulonglong], C.c_int),
    "lbm_cg_create_from_input_seeded": ([C.c_char_p, C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p), C.POINTER(CGInput)],
                                        C.c_int),
    "lbm_cg_mixture_phase": ([_U8P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _F64P], C.c_int),
    "lbm_read_cg_input": ([C.c_char_p, C.POINTER(CGInput)], C.c_int),
    "lbm_read_phase": ([C.c_char_p, C.c_int, C.c_int, C.c_int, _F64P], C.c_int),
    "lbm_cg_create_from_input": ([C.c_char_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(CGInput)], C.c_int),
    "lbm_cg_write_vtk_velocity": ([C.c_void_p, C.c_char_p], C.c_int),
    "lbm_cg_write_vtk_density": ([C.c_void_p, C.c_char_p], C.c_int),
    "lbm_cg_write_vtk_psi": ([C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p], C.c_int),
    "lbm_cg_write_checkpoint": ([C.c_void_p, C.c_char_p, C.c_longlong], C.c_int),
    "lbm_cg_read_checkpoint": ([C.c_void_p, C.c_char_p, C.c_longlong], C.c_int),
    "lbm_st7_create": ([C.c_void_p, _U8P, C.c_int, C.c_int, C.c_int, _F64P, _F64P, C.POINTER(C.c_void_p)], C.c_int),
    "lbm_st7_create_from_flow": ([C.c_void_p, C.c_void_p, _F64P, C.POINTER(C.c_void_p)], C.c_int),
    "lbm_st19_create": ([C.c_void_p, _U8P, C.c_int, C.c_int, C.c_int, _F64P, _F64P, C.POINTER(C.c_void_p)], C.c_int),
    "lbm_st19_create_from_flow": ([C.c_void_p, C.c_void_p, _F64P, C.POINTER(C.c_void_p)], C.c_int),
    "lbm_st7_directions": ([C.c_void_p], C.c_int),
    "lbm_st7_set_lattice": ([C.c_void_p, C.c_double, C.c_double], C.c_int),
    "lbm_st7_step": ([C.c_void_p, C.c_int], C.c_int),
    "lbm_st7_get_concentration": ([C.c_void_p, _F64P], C.c_int),
    "lbm_st7_info": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_double)], C.c_int),
    "lbm_st7_destroy": ([C.c_void_p], None),
    "lbm_st7_get_populations": ([C.c_void_p, _F64P], C.c_int),
    "lbm_st7_set_state": ([C.c_void_p, _F64P, _F64P], C.c_int),
    "lbm_read_st7_input": ([C.c_char_p, C.POINTER(ST7Input)], C.c_int),
    "lbm_slab_partition": ([_U8P, C.c_int, C.c_int, C.c_int, C.c_int, _I32P], C.c_int),
    "lbm_write_velocity_for_solute": ([C.c_void_p, C.c_char_p], C.c_int),
    "lbm_read_velocity_for_solute": ([C.c_char_p, _U8P, C.c_int, C.c_int, C.c_int, _F64P], C.c_int),
    "lbm_write_velocity_for_solute_ordered": ([C.c_void_p, C.c_char_p, C.c_int], C.c_int),
    "lbm_read_velocity_for_solute_ordered": ([C.c_char_p, _U8P, C.c_int, C.c_int, C.c_int, C.c_int, _F64P], C.c_int),
    "lbm_box_sums": ([C.c_void_p, C.c_int, _I32P, _F64P], C.c_int),
    "lbm_group_perm": ([C.c_void_p, C.c_int, _I32P, _I32P, _I32P, _F64P], C.c_int),
    "lbm_local_perm": ([C.c_void_p, _F64P], C.c_int),
    "lbm_write_vtk_geometry": ([_U8P, C.c_int, C.c_int, C.c_int, C.c_char_p], C.c_int),
    "lbm_write_vtk_velocity": ([C.c_void_p, C.c_char_p], C.c_int),
    "lbm_write_vtk_density": ([C.c_void_p, C.c_char_p], C.c_int),
    "lbm_write_checkpoint": ([C.c_void_p, C.c_char_p, C.c_longlong], C.c_int),
    "lbm_read_checkpoint": ([C.c_void_p, C.c_char_p, C.c_longlong], C.c_int),
}


def write_vtk_geometry(mask, path):
    """LBM_Geometry.vtk of a [nz, ny, nx] mask (non-zero = solid)."""
    m = np.ascontiguousarray(mask != 0, dtype=np.uint8)
    nz, ny, nx = m.shape
    _check(lib().lbm_write_vtk_geometry(m.reshape(-1), nx, ny, nz, os.fsencode(path)))


def write_vtk_velocity(flow, path):
    _check(lib().lbm_write_vtk_velocity(flow._h, os.fsencode(path)))


def write_vtk_density(flow, path):
    _check(lib().lbm_write_vtk_density(flow._h, os.fsencode(path)))


def write_checkpoint(flow, prefix, m):
    """Writes <prefix>LBM_checkpoint_{velocity,rho,f}_<m>.0.bin_input."""
    _check(lib().lbm_write_checkpoint(flow._h, os.fsencode(prefix), int(m)))


def read_checkpoint(flow, prefix, m):
    _check(lib().lbm_read_checkpoint(flow._h, os.fsencode(prefix), int(m)))


def release_cached_memory():
    """Returns the device memory destroyed solvers left cached in the
    process's memory pools to the driver (lbm_release_cached_memory)."""
    _check(lib().lbm_release_cached_memory())


def driver_path(name="lbm_sp"):
    """Path of a command-line driver built beside liblbm.so: ``lbm_sp``
    (single phase), ``lbm_cg`` (colour gradient) or ``lbm_st7`` (solute)."""
    if name not in ("lbm_sp", "lbm_cg", "lbm_st7"):
        raise ValueError(f"unknown driver {name!r}")
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), name)


class ST7Params(C.Structure):
    _fields_ = [("diffusivity", C.c_double), ("precision", C.c_int), ("device", C.c_int)]


class Solute:
    """Passive-scalar solve advected by a fixed velocity field: the D3Q7
    solute program (lattice=7) or the D3Q19 one (lattice=19).

    Either ``u_nodes`` ([(count+1), 3], the order of SinglePhase.fields()) or
    ``flow`` (a SinglePhase whose current velocity is used) must be given."""

    def __init__(self, mask, c0, diffusivity, u_nodes=None, flow=None, precision="f64", device=0, lattice=7):
        if lattice not in (7, 19):
            raise ValueError("lattice is 7 or 19")
        p = ST7Params(float(diffusivity), PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                      int(device))
        c0 = np.ascontiguousarray(c0, dtype=np.float64).reshape(-1)
        h = C.c_void_p()
        L = lib()
        if flow is not None:
            fn = L.lbm_st7_create_from_flow if lattice == 7 else L.lbm_st19_create_from_flow
            _check(fn(C.byref(p), flow._h, c0, C.byref(h)))
        else:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            nz, ny, nx = m.shape
            u = np.ascontiguousarray(u_nodes, dtype=np.float64).reshape(-1)
            fn = L.lbm_st7_create if lattice == 7 else L.lbm_st19_create
            _check(fn(C.byref(p), m.reshape(-1), nx, ny, nz, u, c0, C.byref(h)))
        self._h = h
        self.directions = L.lbm_st7_directions(h)
        c, st, ms = C.c_int(), C.c_longlong(), C.c_double()
        _check(lib().lbm_st7_info(h, C.byref(c), C.byref(st), C.byref(ms)))
        self.count = c.value

    def set_lattice(self, dx, dt):
        """Self-defined lattice velocity (lattice_v, dx, dt): tau_s and the
        D3Q19 equilibrium's c2 = (dx/dt)^2, c4 = c2^2 as the program sets them."""
        _check(lib().lbm_st7_set_lattice(self._h, float(dx), float(dt)))

    def step(self, n=1):
        _check(lib().lbm_st7_step(self._h, int(n)))

    def concentration(self):
        c = np.zeros(self.count + 1)
        _check(lib().lbm_st7_get_concentration(self._h, c))
        return c

    def populations(self):
        """g as the next step reads it, [(count+1), 7] (column 0 unused) or,
        for D3Q19, [(count+1), 19] in the solute program's direction order."""
        g = np.zeros((self.count + 1) * self.directions)
        _check(lib().lbm_st7_get_populations(self._h, g))
        return g.reshape(-1, self.directions)

    def set_state(self, g, c):
        """Restores g [(count+1), 7 or 19] and C [(count+1)]; the next step takes C as given."""
        arr = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        _check(lib().lbm_st7_set_state(self._h, arr(g), arr(c)))

    def last_step_ms(self):
        """Device time of the last step() call in ms (CUDA events on the solver's stream)."""
        c, st, ms = C.c_int(), C.c_longlong(), C.c_double()
        _check(lib().lbm_st7_info(self._h, C.byref(c), C.byref(st), C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_st7_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


SOLUTE_ORDERS = {"slab": 0, "xfast": 1}


def write_velocity_for_solute(flow, path, order="slab"):
    """Velocity_for_solute file; ``order`` "slab" is what the solute programs
    read, "xfast" what the 3-D partition program writes."""
    _check(lib().lbm_write_velocity_for_solute_ordered(flow._h, os.fsencode(path), SOLUTE_ORDERS[order]))


def read_velocity_for_solute(path, mask, order="slab"):
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    nz, ny, nx = m.shape
    count = int((m == 0).sum())
    u = np.zeros((count + 1) * 3)
    _check(lib().lbm_read_velocity_for_solute_ordered(os.fsencode(path), m.reshape(-1), nx, ny, nz,
                                                      SOLUTE_ORDERS[order], u))
    return u.reshape(-1, 3)


class ColourGradient:
    """Colour-gradient two-phase solve (periodic) on one GPU.

    ``psi`` holds the initial phase per cell, (nz, ny, nx), +1 = component r.
    ``boundary`` (a ``Boundary``) adds pressure/velocity faces."""

    def __init__(self, mask, psi, nu_l=0.1, nu_g=0.1, psi_solid=0.70711, cap_a=1e-3, g=(1e-5, 0.0, 0.0),
                 body_force_phase=-1, flux_psi=0.99, flux_umax=0.01, precision="f32", device=0, perdir=1,
                 boundary=None):
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        nz, ny, nx = m.shape
        p = CGParams(float(nu_l), float(nu_g), float(psi_solid), float(cap_a), float(g[0]), float(g[1]), float(g[2]),
                     int(body_force_phase), float(flux_psi), float(flux_umax),
                     PRECISIONS[precision] if isinstance(precision, str) else int(precision), int(device), int(perdir))
        h = C.c_void_p()
        _check(lib().lbm_cg_create_bc(C.byref(p), C.byref(boundary) if boundary is not None else None, m.reshape(-1),
                                      np.ascontiguousarray(psi, dtype=np.float64).reshape(-1), nx, ny, nz,
                                      C.byref(h)))
        self._h = h
        c, ph, st, ms = C.c_int(), C.c_double(), C.c_longlong(), C.c_double()
        _check(lib().lbm_cg_info(h, C.byref(c), C.byref(ph), C.byref(st), C.byref(ms)))
        self.count, self.porosity = c.value, ph.value

    @classmethod
    def from_input(cls, input_path, precision="f64", seed=0):
        """Solver of the colour-gradient program's INPUT file (geometry and
        phase file read from the paths it names); returns (solver, input dict).
        seed: the random initial phase and random phase faces."""
        self = cls.__new__(cls)
        h, inp = C.c_void_p(), CGInput()
        _check(lib().lbm_cg_create_from_input_seeded(os.fsencode(input_path),
                                                     PRECISIONS[precision] if isinstance(precision, str)
                                                     else int(precision), int(seed), C.byref(h), C.byref(inp)))
        self._h = h
        c, ph, st, ms = C.c_int(), C.c_double(), C.c_longlong(), C.c_double()
        _check(lib().lbm_cg_info(h, C.byref(c), C.byref(ph), C.byref(st), C.byref(ms)))
        self.count, self.porosity = c.value, ph.value
        return self, inp.as_dict()

    def set_body_force(self, g, before_collision=False):
        """New body force; with before_collision the last step's macro values
        keep the old one (the stabiliser's switch), else they take the new one
        (the force ramps)."""
        _check(lib().lbm_cg_set_body_force(self._h, float(g[0]), float(g[1]), float(g[2]), int(bool(before_collision))))

    def set_cap_a(self, cap_a):
        _check(lib().lbm_cg_set_cap_a(self._h, float(cap_a)))

    def set_initial_velocity(self, u0):
        """Start from feq(1, u0) with u = u0 in the first collision (inivx..z,
        CG3:2357-2400); only before the first step."""
        _check(lib().lbm_cg_set_initial_velocity(self._h, float(u0[0]), float(u0[1]), float(u0[2])))

    def input_update(self, path):
        """input_update (CG3:5765-5925): the INPUT file at `path` read again;
        its wall colour, CapA and flux thresholds apply from the next
        collision, its body force from this step's macro step.  Returns the
        file as a dict (n_max, the output intervals and the permeability are
        the caller's)."""
        inp = CGInput()
        _check(lib().lbm_read_cg_input(os.fsencode(path), C.byref(inp)))
        _check(lib().lbm_cg_input_update(self._h, C.byref(inp)))
        return inp.as_dict()

    def set_faces(self, rho, vel, active=True):
        """Face densities and normal velocities (xp, xn, yp, yn, zp, zn) and
        whether the face rules run; a change acts on the step just run."""
        arr = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(6)
        _check(lib().lbm_cg_set_faces(self._h, arr(rho), arr(vel), int(bool(active))))

    def set_window(self, window, restrict_nodes=True):
        """window = (xn, xp, yn, yp, zn, zp) inclusive, or None for the whole box."""
        w = np.full(6, -1, dtype=np.int32) if window is None else np.ascontiguousarray(window, dtype=np.int32)
        _check(lib().lbm_cg_set_window(self._h, w, int(bool(restrict_nodes))))

    def set_phase_faces(self, faces):
        """Constant initial phase on the box faces (xp, xn, yp, yn, zp, zn; 1 = on)."""
        _check(lib().lbm_cg_set_phase_faces(self._h, np.ascontiguousarray(faces, dtype=np.int32)))

    def set_random(self, ini_sat, seed):
        """Threshold and seed of the random phase faces (face flag 3) for the
        next set_phase_faces."""
        _check(lib().lbm_cg_set_random(self._h, float(ini_sat), int(seed)))

    def set_zero_sigma(self, x_last):
        """Mixture injection: no surface tension in the layer x <= x_last (-1 = off)."""
        _check(lib().lbm_cg_set_zero_sigma(self._h, int(x_last)))

    def set_state(self, f, psi, rho_r, rho_b):
        """Restores f [(count+1), 19] (CG velocity order) and psi / rho_r /
        rho_b [(count+1)], reference id order."""
        arr = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        _check(lib().lbm_cg_set_state(self._h, arr(f), arr(psi), arr(rho_r), arr(rho_b)))

    def write_vtk_velocity(self, path):
        _check(lib().lbm_cg_write_vtk_velocity(self._h, os.fsencode(path)))

    def write_vtk_density(self, path):
        _check(lib().lbm_cg_write_vtk_density(self._h, os.fsencode(path)))

    def write_vtk_psi(self, path, version_suffix="", title=""):
        _check(lib().lbm_cg_write_vtk_psi(self._h, os.fsencode(path), version_suffix.encode(), title.encode()))

    def write_checkpoint(self, prefix, m):
        _check(lib().lbm_cg_write_checkpoint(self._h, os.fsencode(prefix), int(m)))

    def read_checkpoint(self, prefix, m):
        _check(lib().lbm_cg_read_checkpoint(self._h, os.fsencode(prefix), int(m)))

    def step(self, n=1):
        _check(lib().lbm_cg_step(self._h, int(n)))

    def reduce(self):
        d = CGDiag()
        _check(lib().lbm_cg_reduce(self._h, C.byref(d)))
        return d.as_dict()

    def fields(self):
        n = self.count + 1
        out = {"rho": np.zeros(n), "u": np.zeros(n * 3), "psi": np.zeros(n), "rho_r": np.zeros(n),
               "rho_b": np.zeros(n)}
        _check(lib().lbm_cg_get_fields(self._h, out["rho"].ctypes.data, out["u"].ctypes.data, out["psi"].ctypes.data,
                                       out["rho_r"].ctypes.data, out["rho_b"].ctypes.data))
        out["u"] = out["u"].reshape(-1, 3)
        return out

    def populations(self):
        f = np.zeros((self.count + 1) * 19)
        _check(lib().lbm_cg_get_populations(self._h, f))
        return f.reshape(-1, 19)

    def last_step_ms(self):
        c, ph, st, ms = C.c_int(), C.c_double(), C.c_longlong(), C.c_double()
        _check(lib().lbm_cg_info(self._h, C.byref(c), C.byref(ph), C.byref(st), C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_cg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _instance(mask, nu, g):
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    nz, ny, nx = m.shape
    inst = Instance(m.ctypes.data, nx, ny, nz, float(nu), float(g[0]), float(g[1]), float(g[2]))
    return inst, m


class Batch:
    """Many independent single-phase solves in one node pool on one GPU.

    ``solves`` is a list of (mask, nu, g) tuples."""

    def __init__(self, solves, precision="f32", ordering="reference", block=256, device=0):
        keep = []
        arr = (Instance * len(solves))()
        for i, (mask, nu, g) in enumerate(solves):
            arr[i], m = _instance(mask, nu, g)
            keep.append(m)
        h = C.c_void_p()
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        order = ORDERINGS[ordering] if isinstance(ordering, str) else int(ordering)
        _check(lib().lbm_batch_create(len(solves), arr, prec, order, int(block), int(device), C.byref(h)))
        self._h = h
        self.n = len(solves)
        self.counts = None

    def run(self, tol=1e-6, check_every=100, max_steps=1_000_000):
        res = (SolveResult * self.n)()
        _check(lib().lbm_batch_run(self._h, float(tol), int(check_every), int(max_steps), res))
        out = [r.as_dict() for r in res]
        self.counts = [r["count"] for r in out]
        return out

    def reset(self):
        _check(lib().lbm_batch_reset(self._h))

    def fields(self, i):
        if self.counts is None:
            raise LbmError(-8, "run the batch before reading fields")
        n = self.counts[i]
        rho = np.zeros(n + 1)
        u = np.zeros((n + 1) * 3)
        _check(lib().lbm_batch_get_fields(self._h, int(i), rho.ctypes.data, u.ctypes.data))
        return rho, u.reshape(-1, 3)

    def autotune(self, trial_steps=20):
        o, b, m = C.c_int(), C.c_int(), C.c_double()
        _check(lib().lbm_batch_autotune(self._h, int(trial_steps), C.byref(o), C.byref(b), C.byref(m)))
        return {"ordering": o.value, "block": b.value, "mlups": m.value}

    def info(self):
        t, ms, ns = C.c_longlong(), C.c_double(), C.c_longlong()
        _check(lib().lbm_batch_info(self._h, C.byref(t), C.byref(ms), C.byref(ns)))
        return {"total_nodes": t.value, "last_run_ms": ms.value, "node_steps": ns.value}

    def trace(self):
        """Per chain of the last run: [stepping fluid nodes, steps, device ms]."""
        n = C.c_int()
        _check(lib().lbm_batch_trace(self._h, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 3))
        _check(lib().lbm_batch_trace(self._h, out.ctypes.data, n.value, C.byref(n)))
        return out[: n.value]

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """Continuous-batching permeability solve server on one GPU."""

    def __init__(self, capacity_nodes=64 * 1024 * 1024, max_active=256, precision="f32", ordering="reference",
                 block=256, tol=1e-6, check_every=100, max_steps=1_000_000, device=0, target_active_nodes=0,
                 policy="fifo"):
        c = ServerConfig()
        lib().lbm_server_config_default(C.byref(c))
        c.policy = {"fifo": 0, "shortest": 1}[policy] if isinstance(policy, str) else int(policy)
        c.target_active_nodes = int(target_active_nodes)
        c.capacity_nodes = int(capacity_nodes)
        c.max_active = int(max_active)
        c.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        c.ordering = ORDERINGS[ordering] if isinstance(ordering, str) else int(ordering)
        c.block = int(block)
        c.tol = float(tol)
        c.check_every = int(check_every)
        c.max_steps = int(max_steps)
        c.device = int(device)
        h = C.c_void_p()
        _check(lib().lbm_server_create(C.byref(c), C.byref(h)))
        self._h = h

    def submit(self, mask, nu, g):
        inst, m = _instance(mask, nu, g)
        rid = C.c_longlong()
        _check(lib().lbm_server_submit(self._h, C.byref(inst), C.byref(rid)))
        return rid.value

    def pump(self):
        a, q = C.c_int(), C.c_int()
        _check(lib().lbm_server_pump(self._h, C.byref(a), C.byref(q)))
        return a.value, q.value

    def poll(self, max_results=1024):
        buf = (ServerResult * max_results)()
        n = C.c_int()
        _check(lib().lbm_server_poll(self._h, buf, max_results, C.byref(n)))
        out = []
        for r in buf[:n.value]:
            d = r.result.as_dict()
            d.update(request_id=r.request_id, t_submit=r.t_submit, t_admit=r.t_admit, t_done=r.t_done)
            out.append(d)
        return out

    def now(self):
        return lib().lbm_server_now(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().lbm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def lib():
    """Loads liblbm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python jianhui-lbm_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def _check(status):
    if status != 0:
        raise LbmError(status, lib().lbm_last_error().decode(errors="replace"))


def read_input(path):
    """INPUT.dat of the single-phase solvers as a dict (field order SP3:283-340)."""
    out = Input()
    _check(lib().lbm_read_input(os.fsencode(path), C.byref(out)))
    return out.as_dict()


def read_cg_input(path):
    """INPUT file of the colour-gradient program as a dict (field order CG3:372-474)."""
    out = CGInput()
    _check(lib().lbm_read_cg_input(os.fsencode(path), C.byref(out)))
    return out.as_dict()


def read_st7_input(path):
    """INPUT file of the solute program as a dict (field order ST7:219-280)."""
    out = ST7Input()
    _check(lib().lbm_read_st7_input(os.fsencode(path), C.byref(out)))
    return out.as_dict()


def slab_partition(mask, nranks):
    """x-slab split of the slab programs (ST7:951-975) of a [nz, ny, nx] mask:
    rank r holds the x-planes first[r] .. first[r+1]-1."""
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    nz, ny, nx = m.shape
    first = np.zeros(int(nranks) + 1, dtype=np.int32)
    _check(lib().lbm_slab_partition(m.reshape(-1), nx, ny, nz, int(nranks), first))
    return first


def mixture_phase(mask, thickness, portion):
    """Initial phase of the mixture injection (psi_mixture_ini) of a
    [nz, ny, nx] mask: +1 / -1 per cell, [nz, ny, nx] float64."""
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    nz, ny, nx = m.shape
    out = np.zeros(m.size)
    _check(lib().lbm_cg_mixture_phase(m.reshape(-1), nx, ny, nz, int(thickness), float(portion), out))
    return out.reshape(nz, ny, nx)


def read_phase(path, shape):
    """Phase file (x fastest, each value read as float) as [nz, ny, nx] float64."""
    nx, ny, nz = shape
    out = np.zeros(nx * ny * nz)
    _check(lib().lbm_read_phase(os.fsencode(path), nx, ny, nz, out))
    return out.reshape(nz, ny, nx)


def read_mask(path, shape, decbin):
    nx, ny, nz = shape
    m = np.zeros(nx * ny * nz, dtype=np.uint8)
    _check(lib().lbm_read_mask(os.fsencode(path), nx, ny, nz, int(decbin), m))
    return m.reshape(nz, ny, nx)


def default_params():
    p = Params()
    lib().lbm_params_default(C.byref(p))
    return p


class SinglePhase:
    """One single-phase periodic solve resident on a GPU.

    ``mask`` is a (nz, ny, nx) uint8 array, 0 = pore.  ``g`` is the body
    force (acceleration), ``nu`` the kinematic viscosity (tau = 3 nu + 1/2).
    """

    def __init__(self, mask, nu, g=(1e-6, 0.0, 0.0), precision="f32", ordering="reference",
                 block_size=256, u_init=(0.0, 0.0, 0.0), perdir=1, window=None, fp16_scale=0.0, device=0,
                 bc=None, _handle=None):
        self._h = None
        if _handle is not None:
            self._h = _handle
            self._load_info()
            return
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        nz, ny, nx = mask.shape
        p = default_params()
        p.nu = float(nu)
        p.gx, p.gy, p.gz = (float(x) for x in g)
        p.u_init = (C.c_double * 3)(*[float(x) for x in u_init])
        p.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p.ordering = ORDERINGS[ordering] if isinstance(ordering, str) else int(ordering)
        p.block_size = int(block_size)
        p.perdir = int(perdir)
        if window is not None:
            p.window = (C.c_int * 6)(*[int(x) for x in window])
        p.fp16_scale = float(fp16_scale)
        p.device = int(device)
        if bc is not None:
            p.bc = bc if isinstance(bc, Boundary) else Boundary.make(**bc)
        h = C.c_void_p()
        _check(lib().lbm_create(C.byref(p), mask.reshape(-1), nx, ny, nz, C.byref(h)))
        self._h = h
        self.shape = (nx, ny, nz)
        self._load_info()

    @classmethod
    def from_input(cls, input_path, precision="f32", ordering="reference"):
        h = C.c_void_p()
        parsed = Input()
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        order = ORDERINGS[ordering] if isinstance(ordering, str) else int(ordering)
        _check(lib().lbm_create_from_input(os.fsencode(input_path), prec, order, C.byref(h), C.byref(parsed)))
        obj = cls(None, 0, _handle=h)
        obj.input = parsed.as_dict()
        obj.shape = (parsed.nx, parsed.ny, parsed.nz)
        return obj

    def _load_info(self):
        c = C.c_int()
        ph = C.c_double()
        st = C.c_longlong()
        _check(lib().lbm_info(self._h, C.byref(c), C.byref(ph), C.byref(st)))
        self.count = c.value
        self.porosity = ph.value

    @property
    def steps_done(self):
        c = C.c_int()
        ph = C.c_double()
        st = C.c_longlong()
        _check(lib().lbm_info(self._h, C.byref(c), C.byref(ph), C.byref(st)))
        return st.value

    def close(self):
        if self._h:
            lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, n=1):
        _check(lib().lbm_step(self._h, int(n)))

    def reduce(self):
        d = Diag()
        _check(lib().lbm_reduce(self._h, C.byref(d)))
        return d.as_dict()

    def run_to_convergence(self, tol=1e-6, check_every=100, max_steps=100000, raise_on_cap=False):
        d = Diag()
        st = lib().lbm_run_to_convergence(self._h, float(tol), int(check_every), int(max_steps), C.byref(d))
        if st != 0 and (raise_on_cap or st != -6):
            _check(st)
        out = d.as_dict()
        out["status"] = st
        return out

    def fields(self):
        rho = np.zeros(self.count + 1)
        u = np.zeros((self.count + 1) * 3)
        _check(lib().lbm_get_fields(self._h, rho.ctypes.data, u.ctypes.data))
        return rho, u.reshape(-1, 3)

    def box_sums(self, boxes):
        """[(xn, xp, yn, yp, zn, zp), ...] -> array [nbox, 4]: sum u_x, u_y, u_z, pore cells."""
        b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int32).reshape(-1, 6))
        out = np.zeros(b.shape[0] * 4)
        _check(lib().lbm_box_sums(self._h, b.shape[0], b.reshape(-1), out))
        return out.reshape(-1, 4)

    def group_perm(self, n_sub, size, corner):
        """Comput_Grop_Perm: per cube (perm_x, perm_y, perm_z, porosity), divisions concatenated."""
        n_sub = np.ascontiguousarray(n_sub, dtype=np.int32)
        size = np.ascontiguousarray(size, dtype=np.int32)
        corner = np.ascontiguousarray(np.asarray(corner, dtype=np.int32).reshape(-1))
        ncube = int((n_sub.astype(np.int64) ** 3).sum())
        out = np.zeros(max(ncube, 1) * 4)
        _check(lib().lbm_group_perm(self._h, n_sub.size, n_sub, size, corner, out))
        return out[: ncube * 4].reshape(-1, 4)

    def local_perm(self):
        out = np.zeros(3)
        _check(lib().lbm_local_perm(self._h, out))
        return out

    def populations(self):
        f = np.zeros((self.count + 1) * 19)
        _check(lib().lbm_get_populations(self._h, f))
        return f.reshape(-1, 19)

    def set_state(self, rho, u, f):
        _check(lib().lbm_set_state(self._h, np.ascontiguousarray(rho, dtype=np.float64).reshape(-1),
                                   np.ascontiguousarray(u, dtype=np.float64).reshape(-1),
                                   np.ascontiguousarray(f, dtype=np.float64).reshape(-1)))

    def compaction(self):
        c = np.zeros(self.count + 1, dtype=np.int32)
        _check(lib().lbm_export_compaction(self._h, c))
        return c

    def table(self):
        t = np.zeros((self.count + 1) * 19, dtype=np.int32)
        _check(lib().lbm_export_table(self._h, t))
        return t.reshape(-1, 19)

    def autotune(self, trial_steps=20):
        o = C.c_int()
        b = C.c_int()
        m = C.c_double()
        _check(lib().lbm_autotune(self._h, int(trial_steps), C.byref(o), C.byref(b), C.byref(m)))
        return {"ordering": o.value, "block": b.value, "mlups": m.value}

    def last_step_ms(self):
        v = C.c_double()
        _check(lib().lbm_last_step_ms(self._h, C.byref(v)))
        return v.value

    def set_lattice(self, dx, dt):
        """Self-defined lattice velocity (lattice_v, dx, dt): lat_c = dx/dt,
        tau = nu / (c_s^2 dt) + 1/2 with c_s^2 = lat_c^2 / 3.  Before the
        first step; the state restarts from the initial equilibrium."""
        _check(lib().lbm_set_lattice(self._h, float(dx), float(dt)))

    def set_table_mode(self, compact):
        """1: compact pull table (default), 0: the int32 table; identical results."""
        _check(lib().lbm_set_table_mode(self._h, int(compact)))

    def table_info(self):
        c, b, w = C.c_int(), C.c_double(), C.c_double()
        _check(lib().lbm_table_info(self._h, C.byref(c), C.byref(b), C.byref(w)))
        return {"compact": c.value, "table_bytes_per_node": b.value, "wide_fraction": w.value}

    def memory(self):
        b = C.c_size_t()
        bl = C.c_double()
        _check(lib().lbm_memory(self._h, C.byref(b), C.byref(bl)))
        return {"device_bytes": b.value, "bytes_per_lu": bl.value}
