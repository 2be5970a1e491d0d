"""ctypes binding of libcamr_b200.so (the C ABI of include/camr_b200.h).

The shared library is built in-tree (camr_b200/_lib/) by camr_b200.build.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# CAMR_B200_LIB selects another build of the library (e.g. a tuning variant).
LIB_PATH = os.environ.get("CAMR_B200_LIB") or os.path.join(HERE, "_lib", "libcamr_b200.so")

NVAR = 10
# camr_clean_state_parts parts (include/camr_b200.h)
CLEAN_VALID, CLEAN_GHOSTS_FROM_OWNERS, CLEAN_GHOSTS_TEMP, CLEAN_VALID_TEMP = 1, 2, 4, 8
STATUS = {0: "CAMR_OK", 1: "CAMR_ERR_INVALID", 2: "CAMR_ERR_UNSUPPORTED", 3: "CAMR_ERR_CUDA",
          4: "CAMR_ERR_NUMERIC", 5: "CAMR_ERR_NOMEM", 6: "CAMR_ERR_TIMEOUT"}

# Boundary-condition words (Source/Utils/IndexDefines.H:7-12).
BC = {"Interior": 0, "Inflow": 1, "Outflow": 2, "Symmetry": 3, "SlipWall": 4, "NoSlipWall": 5}


class CamrError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)}")


class HydroParams(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "do_mol", "ppm_type", "plm_iorder", "use_pslope", "use_flattening",
        "transverse_reset_density", "dual_energy_update_E_from_e", "allow_negative_energy",
        "allow_small_energy", "add_grav_src", "riemann_solver", "eb_weights_type")] + [
        (n, C.c_double) for n in (
            "difmag", "small", "small_dens", "small_temp", "small_pres", "dual_energy_eta1",
            "dual_energy_eta2", "const_grav", "cfl", "init_shrink", "change_max", "fixed_dt",
            "initial_dt", "max_dt", "eos_gamma", "smallu", "small_num")]


class Fab(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("lo", C.c_int * 3), ("hi", C.c_int * 3),
                ("jstride", C.c_int64), ("kstride", C.c_int64), ("nstride", C.c_int64),
                ("ncomp", C.c_int), ("pad0", C.c_int)]


class Geom(C.Structure):
    _fields_ = [("dom_lo", C.c_int * 3), ("dom_hi", C.c_int * 3), ("is_periodic", C.c_int * 3),
                ("bc_lo", C.c_int * 3), ("bc_hi", C.c_int * 3), ("pad0", C.c_int),
                ("dx", C.c_double * 3), ("prob_lo", C.c_double * 3)]


class BoxTask(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("uin", Fab), ("src", Fab),
                ("dsdt", Fab), ("flx", Fab * 3)]


class EBGeom(C.Structure):
    _fields_ = [("flag", C.c_void_p), ("vfrac", C.c_void_p), ("ap", C.c_void_p * 3),
                ("fc", C.c_void_p * 3), ("g_lo", C.c_int * 3), ("g_hi", C.c_int * 3),
                ("cent", C.c_void_p)]


class BoxFab(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("fab", Fab)]


class LevelDesc(C.Structure):
    _fields_ = [("geom", Geom), ("max_grid_size", C.c_int * 3), ("use_graph", C.c_int)]


class ErrorInfo(C.Structure):
    _fields_ = [("code", C.c_int), ("i", C.c_int), ("j", C.c_int), ("k", C.c_int)]


_lib = None

# Every entry point of include/camr_b200.h with its ctypes signature.
SIGNATURES = {
    "camr_default_params": (None, [C.POINTER(HydroParams)]),
    "camr_version": (C.c_char_p, []),
    "camr_hydro_umdrv": (C.c_int, [C.POINTER(C.c_int * 3), C.POINTER(C.c_int * 3),
                                   C.POINTER(Geom), C.POINTER(Fab), C.POINTER(Fab),
                                   C.POINTER(Fab), C.POINTER(Fab), C.POINTER(Fab),
                                   C.POINTER(Fab), C.POINTER(HydroParams), C.c_double,
                                   C.c_void_p]),
    "camr_hydro_umdrv_full": (C.c_int, [C.POINTER(C.c_int * 3), C.POINTER(C.c_int * 3),
                                        C.POINTER(Geom), C.POINTER(Fab), C.POINTER(Fab),
                                        C.POINTER(Fab), C.POINTER(Fab), C.POINTER(Fab),
                                        C.POINTER(Fab), C.POINTER(Fab), C.POINTER(Fab),
                                        C.POINTER(Fab), C.POINTER(Fab), C.POINTER(Fab),
                                        C.POINTER(Fab), C.POINTER(HydroParams), C.c_double,
                                        C.c_void_p]),
    "camr_level_create": (C.c_int, [C.POINTER(LevelDesc), C.POINTER(HydroParams), C.c_void_p,
                                    C.POINTER(C.c_void_p)]),
    "camr_level_destroy": (C.c_int, [C.c_void_p]),
    "camr_level_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "camr_level_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "camr_level_init_finalize": (C.c_int, [C.c_void_p]),
    "camr_level_advance": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "camr_level_last_dt": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "camr_level_est_dt": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "camr_level_state_fab": (C.c_int, [C.c_void_p, C.POINTER(Fab)]),
    "camr_level_get_error": (C.c_int, [C.c_void_p, C.POINTER(ErrorInfo)]),
    "camr_level_floor_resets": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "camr_fill_ghosts": (C.c_int, [C.POINTER(Geom), C.c_int, C.POINTER(BoxFab), C.c_int,
                                   C.c_void_p]),
    "camr_clean_state": (C.c_int, [C.POINTER(Geom), C.c_int, C.POINTER(BoxFab), C.c_int,
                                   C.POINTER(HydroParams), C.c_void_p]),
    "camr_clean_state_parts": (C.c_int, [C.POINTER(Geom), C.c_int, C.POINTER(BoxFab), C.c_int,
                                         C.POINTER(HydroParams), C.c_int, C.c_void_p]),
    "camr_est_dt": (C.c_int, [C.POINTER(Geom), C.c_int, C.POINTER(BoxFab),
                              C.POINTER(HydroParams), C.POINTER(C.c_double), C.c_void_p]),
    "camr_get_error": (C.c_int, [C.c_void_p, C.POINTER(ErrorInfo)]),
    "camr_level_restart": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "camr_amr_restart": (C.c_int, [C.c_void_p, C.POINTER(C.c_double * 4), C.c_int]),
    "camr_eb_level_floor_resets": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "camr_amr_floor_resets": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "camr_check_rn_div": (C.c_int, [C.c_int64, C.c_uint64, C.POINTER(C.c_int64), C.c_void_p]),
    "camr_write_checkpoint": (C.c_int, [C.c_char_p, C.POINTER(Geom), C.POINTER(C.c_double * 3),
                                        C.POINTER(C.c_double * 2), C.POINTER(C.c_double * 2),
                                        C.POINTER(C.c_int * 2), C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_double]),
    "camr_read_checkpoint": (C.c_int, [C.c_char_p, C.POINTER(Geom), C.POINTER(C.c_double * 2),
                                       C.POINTER(C.c_double * 2), C.POINTER(C.c_int * 2),
                                       C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "camr_launch_count": (C.c_int64, []),
    "camr_level_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "camr_last_error_string": (C.c_char_p, []),
    "camr_level_profile_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_float),
                                          C.POINTER(C.c_char_p), C.c_int,
                                          C.POINTER(C.c_int)]),
    "camr_level_kernels_per_step": (C.c_int64, [C.c_void_p]),
    "camr_level_get_state_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "camr_level_sync": (C.c_int, [C.c_void_p]),
    "camr_measure_fp64_peak": (C.c_int, [C.POINTER(C.c_double), C.c_void_p]),
    "camr_hydro_umdrv_noalloc": (C.c_int, [C.POINTER(C.c_int * 3), C.POINTER(C.c_int * 3),
                                           C.POINTER(Geom), C.POINTER(Fab), C.POINTER(Fab),
                                           C.POINTER(Fab), C.POINTER(Fab), C.POINTER(Fab),
                                           C.POINTER(Fab), C.POINTER(HydroParams), C.c_double,
                                           C.c_void_p]),
    "camr_noalloc_last_error": (C.c_char_p, []),
    "camr_batch_create": (C.c_int, [C.c_int, C.POINTER(BoxTask), C.POINTER(Geom),
                                    C.POINTER(HydroParams), C.c_void_p, C.POINTER(C.c_void_p)]),
    "camr_batch_destroy": (C.c_int, [C.c_void_p]),
    "camr_batch_run": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "camr_batch_autotune": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "camr_batch_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint),
                                    C.c_int]),
    "camr_batch_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint),
                                        C.c_int]),
    "camr_hydro_umdrv_batched": (C.c_int, [C.c_int, C.POINTER(BoxTask), C.POINTER(Geom),
                                           C.POINTER(HydroParams), C.c_double, C.c_void_p]),
    "camr_amr_create": (C.c_int, [C.POINTER(LevelDesc), C.c_int, C.c_void_p,
                                  C.POINTER(HydroParams), C.c_void_p, C.POINTER(C.c_void_p)]),
    "camr_amr_destroy": (C.c_int, [C.c_void_p]),
    "camr_amr_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "camr_amr_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "camr_amr_init_finalize": (C.c_int, [C.c_void_p]),
    "camr_amr_advance": (C.c_int, [C.c_void_p, C.c_int]),
    "camr_amr_clock": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "camr_amr_autotune": (C.c_int, [C.c_void_p]),
    "camr_amr_set_fine_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "camr_amr_fine_cells": (C.c_int64, [C.c_void_p]),
    "camr_amr_kernels_per_step": (C.c_int64, [C.c_void_p]),
    "camr_amr_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "camr_amr_get_error": (C.c_int, [C.c_void_p, C.POINTER(ErrorInfo)]),
    "camr_hydro_umdrv_eb": (C.c_int, [C.POINTER(C.c_int * 3), C.POINTER(C.c_int * 3),
                                      C.POINTER(Geom), C.POINTER(Fab), C.POINTER(EBGeom),
                                      C.POINTER(Fab), C.POINTER(Fab), C.POINTER(Fab),
                                      C.POINTER(Fab), C.POINTER(HydroParams), C.c_int,
                                      C.c_double, C.c_void_p]),
    "camr_eb_level_create": (C.c_int, [C.POINTER(LevelDesc), C.POINTER(EBGeom),
                                       C.POINTER(HydroParams), C.c_int, C.c_void_p,
                                       C.POINTER(C.c_void_p)]),
    "camr_eb_level_destroy": (C.c_int, [C.c_void_p]),
    "camr_eb_level_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "camr_eb_level_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "camr_eb_level_init_finalize": (C.c_int, [C.c_void_p]),
    "camr_eb_level_advance": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "camr_eb_level_dts": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int,
                                    C.POINTER(C.c_int)]),
    "camr_eb_level_autotune": (C.c_int, [C.c_void_p]),
    "camr_eb_level_boxes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
    "camr_eb_level_kernels_per_step": (C.c_int64, [C.c_void_p]),
    "camr_eb_level_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "camr_eb_level_get_error": (C.c_int, [C.c_void_p, C.POINTER(ErrorInfo)]),
    "camr_write_plotfile": (C.c_int, [C.c_char_p, C.POINTER(Geom), C.POINTER(C.c_double * 3),
                                      C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_int, C.c_void_p, C.c_void_p]),
    "camr_read_plotfile": (C.c_int, [C.c_char_p, C.POINTER(Geom), C.c_int, C.c_void_p,
                                     C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "camr_write_plotfile_amr": (C.c_int, [C.c_char_p, C.POINTER(Geom),
                                          C.POINTER(C.c_double * 3), C.c_double, C.c_void_p,
                                          C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "camr_read_plotfile_amr": (C.c_int, [C.c_char_p, C.POINTER(Geom), C.c_int, C.c_void_p,
                                         C.c_int, C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_double), C.c_void_p]),
    "camr_io_last_error": (C.c_char_p, []),
    "camr_adjoint_create": (C.c_int, [C.POINTER(Geom), C.POINTER(HydroParams), C.c_int,
                                      C.c_void_p, C.POINTER(C.c_void_p)]),
    "camr_adjoint_destroy": (C.c_int, [C.c_void_p]),
    "camr_adjoint_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_void_p]),
    "camr_adjoint_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "camr_adjoint_dts": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int]),
    "camr_adjoint_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "camr_adjoint_get_error": (C.c_int, [C.c_void_p, C.POINTER(ErrorInfo)]),
}


def lib():
    """Load libcamr_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"camr_b200 native library not built: {LIB_PATH} "
                          "(run `python -c 'import camr_b200.build as b; b.build()'`)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return _lib


def check(status, what):
    if status != 0:
        detail = lib().camr_last_error_string().decode() if status == 3 else ""
        raise CamrError(status, f"{what} {detail}".strip())


def default_params(**overrides):
    p = HydroParams()
    lib().camr_default_params(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p
