"""ctypes declarations of ``include/alebgk.h`` (the library's C-ABI)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libalebgk_b200.so")

c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)

MAX_NEIGH = 128
NOALLOC_MAX_BODIES = 16        # ALEBGK_NOALLOC_MAX_BODIES
NSTAGES = 10
STAGES = ("transport", "particle", "redo", "sigma", "fixup", "mass_sum", "scale_mood",
          "recollide", "mass_end", "step_begin")
OK, EINVAL, ECUDA, ESTATE, ENOMEM, EDEVICE = 0, -1, -2, -3, -4, -5


class Config(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("N", ctypes.c_int), ("Nv", ctypes.c_int),
        ("mls_order", ctypes.c_int), ("precision", ctypes.c_int),
        ("limiter", ctypes.c_int), ("tau_variable", ctypes.c_int),
        ("device", ctypes.c_int),
        ("R", ctypes.c_double), ("tau", ctypes.c_double), ("dHS", ctypes.c_double),
        ("vmin", ctypes.c_double), ("dv", ctypes.c_double), ("radius", ctypes.c_double),
        ("periodic", ctypes.c_int * 3), ("L", ctypes.c_double * 3),
        ("transport", ctypes.c_int), ("particle", ctypes.c_int),
    ]


class Cloud(ctypes.Structure):
    _fields_ = [
        ("xyz", c_double_p), ("meshv", c_double_p), ("wall", c_double_p),
        ("boundary", c_int_p), ("body_id", c_int_p), ("nnb", c_int_p),
        ("nbr", c_int_p), ("g", c_double_p), ("macro", c_double_p),
    ]


class Body(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("rotates", ctypes.c_int), ("size", ctypes.c_double),
                ("state", ctypes.c_double * 32)]


class CkptHeader(ctypes.Structure):
    _fields_ = [("N", ctypes.c_uint64), ("gstride", ctypes.c_uint64), ("step", ctypes.c_uint64),
                ("t", ctypes.c_double), ("dim", ctypes.c_uint32), ("nbodies", ctypes.c_uint32)]


class Diag(ctypes.Structure):
    _fields_ = [("rho_avg", ctypes.c_double), ("KE", ctypes.c_double), ("T_avg", ctypes.c_double),
                ("p_avg", ctypes.c_double), ("mood_count", ctypes.c_int), ("n", ctypes.c_int)]


class FieldsHeader(ctypes.Structure):
    _fields_ = [("magic", ctypes.c_char * 8), ("version", ctypes.c_uint32),
                ("dim", ctypes.c_uint32), ("N", ctypes.c_uint64), ("step", ctypes.c_int64),
                ("t", ctypes.c_double)]


class Counters(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64), ("transport_flags", ctypes.c_int),
        ("positivity_fixes", ctypes.c_int), ("mood_fail", ctypes.c_int),
        ("mls_degenerate", ctypes.c_int),
        ("mass_before", ctypes.c_double), ("mass_after_transport", ctypes.c_double),
        ("mass_scale", ctypes.c_double), ("mass_end", ctypes.c_double),
        ("error_word", ctypes.c_int), ("transport_kernel", ctypes.c_int),
        ("particle_kernel", ctypes.c_int),
    ]


# name -> (restype, argtypes); every exported symbol of include/alebgk.h
SIGNATURES = {
    "alebgk_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "alebgk_last_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "alebgk_upload": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Cloud), ctypes.c_double]),
    "alebgk_upload_state": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p]),
    "alebgk_download_moments": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "alebgk_download_full": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p]),
    "alebgk_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "alebgk_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "alebgk_step_timed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_float)]),
    "alebgk_profile_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_float)]),
    "alebgk_coeff_build": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(Cloud),
                                          ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_coeff_info": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "alebgk_coeff_get": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p, c_int_p,
                                        c_double_p]),
    "alebgk_coeff_free": (None, [ctypes.c_void_p]),
    "alebgk_get_counters": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Counters)]),
    "alebgk_total_mass": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "alebgk_wall_momentum": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "alebgk_device_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                           c_int_p, c_int_p]),
    "alebgk_body_loads": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p,
                                         c_double_p, c_double_p]),
    "alebgk_body_loads_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p,
                                                 c_double_p, c_double_p]),
    "alebgk_body_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Body),
                                        c_double_p, ctypes.c_double, ctypes.c_double]),
    "alebgk_download_geometry": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p,
                                                c_double_p]),
    "alebgk_case_body_shapes": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p, c_double_p]),
    "alebgk_set_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "alebgk_get_launch": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p]),
    "alebgk_set_march_width": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "alebgk_set_nad_floor": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "alebgk_set_residual_speed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "alebgk_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_float)]),
    "alebgk_residual": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "alebgk_residual_interval": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "alebgk_managed_plan": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p, c_double_p]),
    "alebgk_rows_build": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p, c_int_p,
                                         ctypes.c_int, c_double_p,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_upload_rows": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_double_p]),
    "alebgk_rows_free": (None, [ctypes.c_void_p]),
    "alebgk_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_batch_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "alebgk_batch_set_mode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "alebgk_batch_get_mode": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p]),
    "alebgk_batch_set_groups": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "alebgk_batch_set_spin_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "alebgk_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_float)]),
    "alebgk_batch_residuals": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "alebgk_batch_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "alebgk_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "alebgk_case_build_ex": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_checkpoint_header": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(CkptHeader)]),
    "alebgk_checkpoint_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(CkptHeader),
                                              ctypes.POINTER(Cloud), c_int_p,
                                              ctypes.POINTER(Body)]),
    "alebgk_checkpoint_save": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64,
                                              ctypes.c_double, c_double_p, c_int_p, ctypes.c_int,
                                              ctypes.POINTER(Body)]),
    "alebgk_vtk_write_host": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, c_double_p,
                                             c_double_p, c_int_p, ctypes.c_int,
                                             ctypes.c_double]),
    "alebgk_write_vtk": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                        ctypes.c_double]),
    "alebgk_diagnostics_host": (ctypes.c_int, [ctypes.c_int, c_double_p, c_int_p,
                                               ctypes.POINTER(Diag)]),
    "alebgk_diagnostics": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Diag)]),
    "alebgk_write_timeseries": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_double,
                                               ctypes.POINTER(Diag), ctypes.c_int]),
    "alebgk_format_step": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double,
                                          ctypes.POINTER(Diag)]),
    "alebgk_write_fields": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64,
                                           ctypes.c_double]),
    "alebgk_read_fields": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(FieldsHeader),
                                          c_double_p, c_double_p, c_int_p]),
    "alebgk_body_set_surface_velocity": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                                        c_double_p, c_double_p]),
    "alebgk_case_build": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_case_free": (None, [ctypes.c_void_p]),
    "alebgk_case_info": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_double_p]),
    "alebgk_case_view": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Cloud)]),
    "alebgk_case_bodies": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "alebgk_case_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(Config)]),
    "alebgk_lattice_info": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, c_int_p,
                                           c_double_p]),
    "alebgk_lattice_build_device": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_int, c_double_p,
                                                   c_double_p, c_int_p, c_int_p, c_int_p]),
    "alebgk_lattice_info_ex": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                              c_int_p, c_double_p]),
    "alebgk_lattice_bodies": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, c_int_p, c_double_p, c_int_p,
                                             c_int_p, c_double_p]),
    "alebgk_lattice_build_device_ex": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int,
                                                      ctypes.c_int, ctypes.c_double,
                                                      ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_double, ctypes.c_double,
                                                      ctypes.c_double, ctypes.c_double,
                                                      ctypes.c_int, c_double_p, c_double_p,
                                                      c_int_p, c_int_p, c_int_p, c_int_p]),
    "alebgk_upload_lattice_ex": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double]),
    "alebgk_upload_lattice": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double]),
    "alebgk_slab_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                          c_int_p, c_int_p, ctypes.c_int, c_int_p,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_slab_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "alebgk_slab_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "alebgk_slab_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "alebgk_rank_slab_init": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, c_double_p]),
    "alebgk_rank_slab_segment": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p]),
    "alebgk_rank_slab_combine": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                c_double_p]),
    "alebgk_rank_slab_rows": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_void_p, c_double_p, ctypes.c_int]),
    "alebgk_rank_slab_finish": (ctypes.c_int, [ctypes.c_void_p]),
    "alebgk_neighbours_device": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_int_p, c_int_p,
                                                c_int_p]),
    "alebgk_manage_cloud": (ctypes.c_int, [ctypes.c_int, c_double_p, c_int_p, ctypes.c_int,
                                           ctypes.POINTER(Body), ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(Cloud), ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_managed_info": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "alebgk_managed_cloud": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Cloud)]),
    "alebgk_managed_free": (None, [ctypes.c_void_p]),
    "alebgk_upload_geometry": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Cloud),
                                              ctypes.c_double]),
    "alebgk_set_coeff_builder": (ctypes.c_int, [ctypes.c_int]),
    "alebgk_moments13": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "alebgk_seed_grad13": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          c_double_p, c_double_p]),
    "alebgk_net_nparams": (ctypes.c_int, []),
    "alebgk_net_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "alebgk_net_destroy": (None, [ctypes.c_void_p]),
    "alebgk_net_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "alebgk_net_set_params": (ctypes.c_int, [ctypes.c_void_p, c_float_p]),
    "alebgk_net_get_params": (ctypes.c_int, [ctypes.c_void_p, c_float_p]),
    "alebgk_net_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_void_p]),
    "alebgk_net_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_int, c_float_p, c_float_p,
                                       c_float_p]),
    "alebgk_net_train_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int, c_float_p,
                                             ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                             ctypes.c_float, c_float_p]),
    "alebgk_net_sync": (ctypes.c_int, [ctypes.c_void_p]),
}

_lib = None


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads the in-tree library and declares every C-ABI signature.

    Raises if the library is missing: there is no fallback implementation.
    """
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python -m alebgk4paper_b200.build` "
            "(the ALE-BGK step has no CPU fallback)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
