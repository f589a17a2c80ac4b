"""ctypes binding of libsolfec_b200.so (the sm_100a kernels, the device-layer C
ABI of include/b2_device.h and the host C layer of include/solfec_b200.h).

There is no CPU fallback: if the library is missing or fails to load, every
entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, 'lib', 'libsolfec_b200.so')

_lib = None


def build(force: bool = False) -> str:
    """Compile the library in-tree for sm_100a (make -C solfec-1.0_b200)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(['make', '-s', '-C', PKG_ROOT], check=True)
    return LIB_PATH


class b2dev_solve_opts(C.Structure):
    _fields_ = [('epsilon', C.c_double), ('meritval', C.c_double), ('diagepsilon', C.c_double),
                ('maxiter', C.c_int), ('diagmaxiter', C.c_int), ('diagsolver', C.c_int), ('failure', C.c_int),
                ('reverse', C.c_int), ('nomerit', C.c_int), ('precision', C.c_int), ('grid', C.c_int),
                ('stage_blocks', C.c_int)]


class b2dev_solve_report(C.Structure):
    _fields_ = [('iters', C.c_int), ('thrown', C.c_int), ('last_fail_kind', C.c_int), ('nfailures', C.c_int),
                ('sweeps', C.c_int), ('iters_mixed', C.c_int), ('merit', C.c_double), ('error', C.c_double),
                ('merit_input', C.c_double), ('ms_device', C.c_float), ('ms_kernel', C.c_float * 2),
                ('sweeps_launch', C.c_int * 2), ('grid', C.c_int)]


class b2gs_bodies(C.Structure):
    _fields_ = [('nbod', C.c_int), ('rot', C.c_void_p), ('x0', C.c_void_p), ('jinv', C.c_void_p),
                ('minv', C.c_void_p), ('velo', C.c_void_p), ('velo0', C.c_void_p), ('obstacle', C.c_void_p),
                ('on_device', C.c_int)]


class b2gs_contacts(C.Structure):
    _fields_ = [('ncon', C.c_int), ('master', C.c_void_p), ('slave', C.c_void_p), ('mpnt', C.c_void_p),
                ('spnt', C.c_void_p), ('base', C.c_void_p), ('gap', C.c_void_p), ('friction', C.c_void_p),
                ('restitution', C.c_void_p), ('cohesion', C.c_void_p), ('on_device', C.c_int)]


class b2dev_batch_report(C.Structure):
    _fields_ = [('iters', C.c_int), ('thrown', C.c_int), ('last_fail_kind', C.c_int), ('nfailures', C.c_int),
                ('merit', C.c_double), ('error', C.c_double), ('merit_input', C.c_double),
                ('ms_to_decision', C.c_double), ('rows', C.c_int)]


class b2dev_tune_result(C.Structure):
    _fields_ = [('tile_rows', C.c_int), ('grid', C.c_int), ('stage_blocks', C.c_int), ('ntrials', C.c_int),
                ('ms', C.c_float), ('trial_rows', C.c_int * 32), ('trial_grid', C.c_int * 32),
                ('trial_stage', C.c_int * 32), ('trial_ms', C.c_float * 32)]


CALLBACK = C.CFUNCTYPE(None, C.c_void_p)

# exported symbols declared in include/*.h with their ctypes signatures
_SIGNATURES = {
    # include/b2_device.h
    'b2dev_last_error': (C.c_char_p, []),
    'b2dev_create': (C.c_void_p, [C.c_int, C.c_void_p]),
    'b2dev_destroy': (None, [C.c_void_p]),
    'b2dev_stream': (C.c_void_p, [C.c_void_p]),
    'b2dev_upload_scene': (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 7 + [C.c_int] + [C.c_void_p] * 9 + [C.c_int]),
    'b2dev_assemble': (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_uint64]),
    'b2dev_rigid_setup': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_rigid_step_begin': (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_rigid_step_end': (C.c_int, [C.c_void_p, C.c_double]),
    'b2dev_rigid_get': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_update_constraints': (C.c_int, [C.c_void_p]),
    'b2dev_constraints_setup': (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 7),
    'b2dev_spheres_setup': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                      C.c_void_p, C.c_int]),
    'b2dev_detect_spheres': (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    'b2dev_convexes_setup': (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 7),
    'b2dev_rigid_flags': (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_set_kinds': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_exclude_bodies': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    'b2dev_exclude_surfaces': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    'b2dev_unphysical_penetration': (C.c_int, [C.c_void_p, C.c_double]),
    'b2dev_contact_sparsify': (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    'b2dev_get_contact_area': (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_detect_carry_state': (C.c_int, [C.c_void_p]),
    'b2dev_get_contacts': (C.c_int, [C.c_void_p] + [C.c_void_p] * 14 + [C.c_int]),
    'b2dev_sphere_centres': (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_upload_locdyn': (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 12 + [C.c_double, C.c_double, C.c_int,
                                                                                  C.c_uint64, C.c_int]),
    'b2dev_set_state': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_get_state': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    'b2dev_solve': (C.c_int, [C.c_void_p, C.POINTER(b2dev_solve_opts), C.POINTER(b2dev_solve_report), C.c_void_p,
                              C.c_void_p]),
    'b2dev_sizes': (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                              C.POINTER(C.c_double)]),
    'b2dev_get_order': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2dev_get_colours': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2dev_get_locdyn': (C.c_int, [C.c_void_p] + [C.c_void_p] * 8 + [C.POINTER(C.c_double)]),
    'b2dev_last_assemble_ms': (C.c_float, [C.c_void_p]),
    'b2dev_launch_count': (C.c_longlong, [C.c_void_p]),
    'b2dev_colour_noalloc': (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                       C.c_void_p]),
    'b2dev_trace_sweep': (C.c_int, [C.c_void_p, C.c_int]),
    'b2dev_get_trace': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2dev_diag_solve_batch': (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                         C.c_double] + [C.c_void_p] * 11),
    'b2dev_set_colour_order': (C.c_int, [C.c_void_p, C.c_int]),
    'b2dev_colour_reuse_count': (C.c_longlong, [C.c_void_p]),
    'b2dev_set_problems': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    'b2dev_problem_free_energy': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2dev_set_tile_rows': (C.c_int, [C.c_void_p, C.c_int]),
    'b2dev_tile_rows': (C.c_int, [C.c_void_p]),
    'b2dev_set_wait_limit': (C.c_int, [C.c_void_p, C.c_double]),
    'b2dev_solve_batch': (C.c_int, [C.c_void_p, C.POINTER(b2dev_solve_opts), C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.POINTER(b2dev_solve_report), C.c_int]),
    'b2dev_autotune_batch': (C.c_int, [C.c_void_p, C.POINTER(b2dev_solve_opts), C.POINTER(b2dev_tune_result)]),
    'b2dev_mlp_nparams': (C.c_int, []),
    'b2dev_mlp_create': (C.c_int, [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    'b2dev_mlp_destroy': (None, [C.c_void_p]),
    'b2dev_mlp_set_params': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2dev_mlp_get_params': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2dev_mlp_grad': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    'b2dev_mlp_train': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double,
                                  C.c_uint64, C.c_void_p]),
    'b2dev_mlp_forward': (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    'b2dev_nn_features': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    'b2dev_nn_warm_start': (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    # include/solfec_b200.h
    'b2gs_create': (C.c_void_p, [C.c_double, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int,
                                 C.c_void_p, CALLBACK]),
    'b2gs_solve': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2gs_failure_string': (C.c_char_p, [C.c_void_p]),
    'b2gs_diagsolver_string': (C.c_char_p, [C.c_void_p]),
    'b2gs_error_string': (C.c_char_p, [C.c_void_p]),
    'b2gs_reverse_string': (C.c_char_p, [C.c_void_p]),
    'b2gs_variant_string': (C.c_char_p, [C.c_void_p]),
    'b2gs_destroy': (None, [C.c_void_p]),
    'b2gs_write_state': (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    'b2gs_get_iters': (C.c_int, [C.c_void_p]),
    'b2gs_get_error': (C.c_int, [C.c_void_p]),
    'b2gs_get_rerhist': (C.POINTER(C.c_double), [C.c_void_p]),
    'b2gs_get_merhist': (C.POINTER(C.c_double), [C.c_void_p]),
    'b2gs_get_itershist': (C.POINTER(C.c_int), [C.c_void_p, C.POINTER(C.c_int)]),
    'b2gs_set_itershist': (None, [C.c_void_p, C.c_int]),
    'b2gs_set_reverse': (None, [C.c_void_p, C.c_int]),
    'b2gs_set_variant': (None, [C.c_void_p, C.c_int]),
    'b2gs_set_nomerit': (None, [C.c_void_p, C.c_int]),
    'b2gs_set_params': (None, [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int]),
    'b2gs_set_precision': (None, [C.c_void_p, C.c_int]),
    'b2gs_set_grid': (None, [C.c_void_p, C.c_int]),
    'b2gs_set_stage_blocks': (None, [C.c_void_p, C.c_int]),
    'b2gs_get_opts': (C.c_int, [C.c_void_p, C.POINTER(b2dev_solve_opts)]),
    'b2gs_get_iters_mixed': (C.c_int, [C.c_void_p]),
    'b2gs_get_solve_ms': (C.c_double, [C.c_void_p]),
    'b2gs_get_merit_input': (C.c_double, [C.c_void_p]),
    'b2gs_get_report': (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    'b2gs_locdyn_create': (C.c_void_p, [C.c_int, C.c_void_p]),
    'b2gs_locdyn_destroy': (None, [C.c_void_p]),
    'b2gs_locdyn_update_begin_resident': (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    'b2gs_write_w_matrix_market': (C.c_int, [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    'b2gs_locdyn_w_matrix_market': (C.c_int, [C.c_void_p, C.c_char_p]),
    'b2gs_write_locdyn_dump': (C.c_int, [C.c_char_p, C.c_int] + [C.c_void_p] * 12),
    'b2gs_locdyn_dump': (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    'b2gs_locdyn_update_begin': (C.c_int, [C.c_void_p, C.POINTER(b2gs_bodies), C.POINTER(b2gs_contacts),
                                           C.c_double, C.c_int]),
    'b2gs_locdyn_set': (C.c_int, [C.c_void_p, C.c_int] + [C.c_void_p] * 12 + [C.c_double, C.c_double, C.c_int,
                                                                              C.c_int]),
    'b2gs_locdyn_set_state': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    'b2gs_locdyn_get_state': (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    'b2gs_locdyn_merit': (C.c_double, [C.c_void_p]),
    'b2gs_locdyn_sizes': (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                    C.POINTER(C.c_double)]),
    'b2gs_locdyn_order': (C.c_int, [C.c_void_p, C.c_void_p]),
    'b2gs_locdyn_set_colour_seed': (None, [C.c_void_p, C.c_uint64]),
    'b2gs_locdyn_device': (C.c_void_p, [C.c_void_p]),
    'b2gs_last_error': (C.c_char_p, []),
}


def lib():
    """The loaded library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError('libsolfec_b200.so not built at %s (run __graft_entry__.build() or make -C %s)'
                               % (LIB_PATH, PKG_ROOT))
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_SIGNATURES)


def last_error() -> str:
    msg = lib().b2gs_last_error()
    return msg.decode() if msg else ''


def ptr(a) -> C.c_void_p:
    """Address of a numpy array (host) or of a torch tensor (device or host)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())
