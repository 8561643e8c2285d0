"""ctypes binding of libdnsb.so (the C ABI declared in include/dnsb.h).

The shared library is built in-tree (see build.py) and loaded from this
package directory.  There is no fallback: if the library is missing or a
symbol is absent, importing the operators fails loudly.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libdnsb.so")

DNSB_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "unsupported size", 4: "out of memory"}

c_double = ctypes.c_double
c_int = ctypes.c_int
c_long = ctypes.c_long
c_void_p = ctypes.c_void_p
P = c_void_p


class dnsb_grid(ctypes.Structure):
    _fields_ = [
        ("nx", c_int), ("ny", c_int), ("nz", c_int),
        ("bc_y", c_int), ("ydiffusion", c_int),
        ("dx", c_double), ("dz", c_double),
        ("dy", P), ("dyu", P),
        ("visc", c_double),
        ("bodyforce", c_double * 3),
    ]


class dnsb_tuning(ctypes.Structure):
    _fields_ = [("lines_x", c_int), ("lines_z", c_int), ("lines_y", c_int), ("lines_z4", c_int),
                ("cell_bx", c_int), ("cell_by", c_int), ("gm_planes", c_int)]


# name -> (restype, argtypes); every symbol declared in include/dnsb.h
SIGNATURES = {
    "dnsb_version": (c_int, []),
    "dnsb_create": (c_int, [ctypes.POINTER(dnsb_grid), c_int, P, ctypes.POINTER(c_void_p)]),
    "dnsb_create_tuned": (c_int, [ctypes.POINTER(dnsb_grid), ctypes.POINTER(dnsb_tuning), c_int, P,
                                  ctypes.POINTER(c_void_p)]),
    "dnsb_get_tuning": (c_int, [P, ctypes.POINTER(dnsb_tuning)]),
    "dnsb_destroy": (None, [P]),
    "dnsb_last_error": (ctypes.c_char_p, [P]),
    "dnsb_set_stream": (c_int, [P, P]),
    "dnsb_sync": (c_int, [P]),
    "dnsb_set_wait_limit": (c_int, [P, ctypes.c_ulong]),
    "dnsb_fill_ghosts": (c_int, [P, P, c_int]),
    "dnsb_divergence": (c_int, [P, P, P, P, P]),
    "dnsb_momentum": (c_int, [P, P, P, P, P, P, P, c_double, c_double]),
    "dnsb_pressuregrad": (c_int, [P, P, P, c_int, c_double]),
    "dnsb_poisson": (c_int, [P, P, P]),
    "dnsb_project": (c_int, [P, P, P, P, P]),
    "dnsb_axpy": (c_int, [P, P, P, c_double]),
    "dnsb_poisson_x": (c_int, [P, P]),
    "dnsb_poisson_zy": (c_int, [P, P, c_int, c_int]),
    "dnsb_poisson_xinv": (c_int, [P, P]),
    "dnsb_spectrum": (c_int, [P, ctypes.POINTER(c_void_p), ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                              ctypes.POINTER(c_int)]),
    "dnsb_zblock_copy": (c_int, [P, P, P, c_int, c_int, c_int, c_int, c_int, c_int, c_int]),
    "dnsb_imex_update": (c_int, [P, P, P, P, P, P, P, P, c_double, c_double, c_double]),
    "dnsb_sfs_stage": (c_int, [P, P, P, P, P, P, P, P, c_double, c_double]),
    "dnsb_step": (c_int, [P, P, P, P, P, P, P, P, P, c_double]),
    "dnsb_cfl": (c_int, [P, P, P, P, c_double, c_int, ctypes.POINTER(c_double)]),
    "dnsb_solve": (c_int, [P, P, P, P, P, P, P, P, P, c_double, c_double, c_double, c_double,
                           c_long, ctypes.POINTER(c_double), ctypes.POINTER(c_long)]),
    "dnsb_solve_host": (c_int, [P, P, P, P, P, c_double, c_double, c_double, c_double, c_long,
                                ctypes.POINTER(c_double), ctypes.POINTER(c_long)]),
    "dnsb_maxdiv": (c_int, [P, P, P, P, ctypes.POINTER(c_double)]),
    "dnsb_kinetic_energy": (c_int, [P, P, P, P, ctypes.POINTER(c_double)]),
    "dnsb_channel_sample": (c_int, [P, P, P, P, P]),
    "dnsb_spectrum_sample": (c_int, [P, P, P, P, P, c_int]),
    "dnsb_noise": (c_int, [P, P, c_int, ctypes.c_ulonglong, c_double]),
    "dnsb_shell_count": (c_int, [P]),
    "dnsb_shell_energies": (c_int, [P, P, P, P, ctypes.POINTER(c_double), c_int]),
    "dnsb_shell_rescale": (c_int, [P, P, P, P, ctypes.POINTER(c_double), c_int]),
    "dnsb_random_field": (c_int, [P, P, P, P, c_double, c_double, ctypes.c_ulonglong,
                                  ctypes.POINTER(c_double), c_int]),
    "dnsb_shell_clamp": (c_int, [P, P, P, P, ctypes.POINTER(c_double), c_int]),
    "dnsb_les_cube": (c_int, [P, P, P, P, c_int, ctypes.POINTER(c_double)]),
    "dnsb_profile": (c_int, [P, c_int]),
    "dnsb_profile_read": (c_int, [P, c_int, ctypes.POINTER(c_double), ctypes.POINTER(c_long)]),
    "dnsb_launch_count": (c_long, [P]),
    "dnsb_kind_name": (ctypes.c_char_p, [c_int]),
    "dnsb_poisson_noalloc": (c_int, [ctypes.POINTER(dnsb_grid), P, P, P]),
    "dnsb_ensemble_create": (c_int, [c_int, ctypes.POINTER(dnsb_grid), c_int, P,
                                     ctypes.POINTER(c_void_p)]),
    "dnsb_ensemble_create_tuned": (c_int, [c_int, ctypes.POINTER(dnsb_grid), ctypes.POINTER(dnsb_tuning),
                                           c_int, P, ctypes.POINTER(c_void_p)]),
    "dnsb_ensemble_destroy": (None, [P]),
    "dnsb_ensemble_last_error": (ctypes.c_char_p, [P]),
    "dnsb_ensemble_member": (P, [P, c_int]),
    "dnsb_ensemble_run": (c_int, [P, ctypes.POINTER(c_void_p), ctypes.POINTER(c_double), c_long]),
    "dnsb_ensemble_forcing": (c_int, [P, c_int, ctypes.POINTER(c_double), c_int]),
    "dnsb_spectral_create": (c_int, [c_int, c_int, c_double, c_double, c_int, P,
                                     ctypes.POINTER(c_void_p)]),
    "dnsb_spectral_destroy": (None, [P]),
    "dnsb_spectral_last_error": (ctypes.c_char_p, [P]),
    "dnsb_spectral_set_stream": (c_int, [P, P]),
    "dnsb_spectral_size": (c_long, [P]),
    "dnsb_spectral_to_phys": (c_int, [P, P, P]),
    "dnsb_spectral_from_phys": (c_int, [P, P, P]),
    "dnsb_spectral_rhs": (c_int, [P, P, P]),
    "dnsb_spectral_project": (c_int, [P, P]),
    "dnsb_spectral_step": (c_int, [P, P, c_double, ctypes.POINTER(c_double)]),
    "dnsb_spectral_vsummax": (c_int, [P, P, ctypes.POINTER(c_double)]),
    "dnsb_spectral_diagnostic": (c_int, [P, P, c_int, ctypes.POINTER(c_double)]),
    "dnsb_spectral_shell_count": (c_int, [P]),
    "dnsb_spectral_shell_energies": (c_int, [P, P, ctypes.POINTER(c_double), c_int]),
    "dnsb_spectral_shell_rescale": (c_int, [P, P, ctypes.POINTER(c_double), c_int]),
    "dnsb_spectral_random_field": (c_int, [P, P, c_double, c_double, ctypes.c_ulonglong,
                                           ctypes.POINTER(c_double), c_int]),
    "dnsb_spectral_shell_clamp": (c_int, [P, P, ctypes.POINTER(c_double), c_int]),
    "dnsb_spectral_les_cube": (c_int, [P, P, c_int, ctypes.POINTER(c_double)]),
    "dnsb_spectral_phaserandomize": (c_int, [P, P, ctypes.c_ulonglong]),
}

# include/dnsb_cnn.h
SIGNATURES.update({
    "dnsb_cnn_create": (c_int, [c_int, P, c_int, c_int, c_int, ctypes.POINTER(c_void_p)]),
    "dnsb_cnn_destroy": (None, [P]),
    "dnsb_cnn_last_error": (ctypes.c_char_p, [P]),
    "dnsb_cnn_set_stream": (c_int, [P, P]),
    "dnsb_cnn_sync": (c_int, [P]),
    "dnsb_cnn_launch_count": (c_long, [P]),
    "dnsb_cnn_param_count": (c_int, [P]),
    "dnsb_cnn_init": (c_int, [P, ctypes.c_ulonglong]),
    "dnsb_cnn_set_params": (c_int, [P, P]),
    "dnsb_cnn_get_params": (c_int, [P, P]),
    "dnsb_cnn_set_scales": (c_int, [P, P, P]),
    "dnsb_cnn_set_dataset": (c_int, [P, P, c_int, c_int]),
    "dnsb_cnn_train": (c_int, [P, c_int, ctypes.c_float, ctypes.c_ulonglong]),
    "dnsb_cnn_steps": (c_int, [P, ctypes.POINTER(c_long)]),
    "dnsb_cnn_losses": (c_int, [P, P, c_long, c_long]),
    "dnsb_cnn_batch": (c_int, [P, P, P, c_int, ctypes.c_float, P, P]),
    "dnsb_cnn_infer_cells": (c_int, [P, P, P]),
    "dnsb_cnn_infer": (c_int, [P, P, P, P, P]),
    "dnsb_les_step": (c_int, [P, P, P, P, P, P, P, P, P, P, c_double]),
    "dnsb_les_advance": (c_int, [P, P, P, P, P, P, P, P, P, P, c_double, c_double, c_double, P, c_int,
                                 ctypes.POINTER(c_double), ctypes.POINTER(c_long)]),
    "dnsb_cnn_profile": (c_int, [P, c_int]),
    "dnsb_cnn_profile_read": (c_int, [P, c_int, ctypes.POINTER(c_double), ctypes.POINTER(c_long),
                                      ctypes.POINTER(c_double)]),
})

KINDS = ["momentum", "cn_solve", "div_rfft_x", "fft_z", "y_solve", "ifft_z", "irfft_x",
         "grad_update", "other", "grad_momentum", "fft_z_y_solve"]

_LIB = None


def load():
    """Load libdnsb.so and bind every entry point (raises if anything is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIBPATH):
        raise ImportError(
            f"{LIBPATH} is missing: build it with `python -m distributednavierstokes_b200.build` "
            "(nvcc, sm_100a); there is no CPU fallback")
    lib = ctypes.CDLL(LIBPATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if the symbol is absent
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class DNSBError(RuntimeError):
    pass


def check(rc, ctx=None):
    if rc != DNSB_OK:
        msg = load().dnsb_last_error(ctx)
        msg = msg.decode() if msg else ""
        raise DNSBError(f"libdnsb: {ERRORS.get(rc, rc)}: {msg}")


def check_cnn(rc, cnn=None):
    if rc != DNSB_OK:
        msg = load().dnsb_cnn_last_error(cnn)
        msg = msg.decode() if msg else ""
        raise DNSBError(f"libdnsb (closure): {ERRORS.get(rc, rc)}: {msg}")
