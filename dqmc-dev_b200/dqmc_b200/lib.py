"""ctypes binding of the engine's C ABI (include/dqmc_b200.h).

The shared library is built in tree (dqmc-dev_b200/lib/libdqmc_b200.so by
`make -C dqmc-dev_b200` or __graft_entry__.build()).  Loading fails loudly
when it is missing: there is no CPU fallback for the engine.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libdqmc_b200.so")

DQMC_OK = 0
DQMC_E_ARG = -10
DQMC_E_CUDA = -11
DQMC_E_NOMEM = -12
DQMC_E_DEVICE = -13
DQMC_E_SCRATCH = -14
NOALLOC_SCRATCH_BYTES = 16 << 20   # DQMC_NOALLOC_SCRATCH_BYTES

# every symbol include/dqmc_b200.h declares
EXPORTS = [
    "dqmc_wrapper", "dqmc_wrapper_batch", "dqmc_acc_sizes", "dqmc_engine_create",
    "dqmc_engine_destroy", "dqmc_engine_set_chain", "dqmc_engine_set_acc",
    "dqmc_engine_init", "dqmc_engine_sweeps", "dqmc_engine_sync", "dqmc_engine_errors",
    "dqmc_engine_get_chain", "dqmc_engine_get_acc", "dqmc_engine_get_g",
    "dqmc_engine_accepts", "dqmc_engine_stream", "dqmc_engine_lanes",
    "dqmc_engine_set_chains", "dqmc_engine_get_chains", "dqmc_engine_launches_per_sweep",
    "dqmc_engine_profile_sweep", "dqmc_engine_profile_grad", "dqmc_engine_update_on_chip",
    "dqmc_engine_logdet_grad",
    "dqmc_engine_obs_grad",
    "dqmc_engine_set_hopping", "dqmc_engine_check_g", "dqmc_engine_g_drift",
    "dqmc_engine_g_drift_ue", "dqmc_engine_g_drift_acc",
    "dqmc_batch_create", "dqmc_batch_sweeps", "dqmc_batch_stream", "dqmc_batch_destroy",
    "dqmc_gpu_gemm", "dqmc_gpu_calc_eq_g", "dqmc_gpu_update_delayed", "dqmc_gpu_mul_seq",
    "dqmc_gpu_calc_eq_g_noalloc",
]


# the measurement toggles and their maps, appended to dqmc_params
TOGGLES = ("meas_energy_corr", "meas_thermal", "meas_2bond_corr", "meas_nematic_corr",
           "meas_chiral", "meas_local_JQ", "meas_gen_suscept", "meas_pair_bb_only")
TOGGLE_INTS = TOGGLES + (
    "Nx", "Ny", "num_plaq", "num_plaq_accum", "num_b_accum", "num_b2_accum",
    "num_bs", "num_b2", "num_b2b", "num_bb2", "num_b2b2",
    "degen_plaq", "degen_b", "degen_b2", "degen_bs", "degen_b2b", "degen_bb2", "degen_b2b2")
TOGGLE_PTRS = ("plaqs", "map_plaq", "map_b", "map_bs", "bond2s", "map_b2", "map_bb2",
               "map_b2b", "map_b2b2", "pp_u", "pp_d", "ppr_u", "ppr_d")


class Params(C.Structure):
    """dqmc_params of include/dqmc_b200.h"""
    _fields_ = (
        [(n, C.c_int) for n in (
            "N", "L", "n_matmul", "n_delay", "F", "n_sweep_warm", "n_sweep",
            "period_eqlt", "period_uneqlt", "meas_bond_corr", "num_i", "num_ij",
            "num_b", "num_bb", "degen_i", "degen_ij", "degen_bb", "cplx")]
        + [(n, C.c_void_p) for n in (
            "map_i", "map_ij", "bonds", "map_bb", "peierlsu", "peierlsd",
            "exp_Ku", "exp_Kd", "inv_exp_Ku", "inv_exp_Kd",
            "exp_halfKu", "exp_halfKd", "inv_exp_halfKu", "inv_exp_halfKd")]
        + [(n, C.c_int) for n in TOGGLE_INTS]
        + [(n, C.c_void_p) for n in TOGGLE_PTRS]
    )


_lib = None


def load(path: str | None = None):
    """Load libdqmc_b200.so (once) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"engine library not built: {p} -- run `make -C dqmc-dev_b200` "
            "(or __graft_entry__.build()); the engine has no CPU fallback")
    lib = C.CDLL(p)
    vp, i, u64p, ip = C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_int)
    sig = {
        "dqmc_wrapper": (i, [C.c_char_p, C.c_char_p, C.c_int64, C.c_bool, C.c_bool]),
        "dqmc_wrapper_batch": (i, [i, C.POINTER(C.c_char_p), C.c_char_p, C.c_int64,
                                   C.c_bool, ip]),
        "dqmc_acc_sizes": (i, [C.POINTER(Params), ip, ip]),
        "dqmc_engine_create": (i, [C.POINTER(Params), i, i, C.POINTER(vp)]),
        "dqmc_engine_destroy": (None, [vp]),
        "dqmc_engine_set_chain": (i, [vp, i, vp, vp, vp, vp, i]),
        "dqmc_engine_set_acc": (i, [vp, i, i, vp, i, vp]),
        "dqmc_engine_init": (i, [vp]),
        "dqmc_engine_sweeps": (i, [vp, i, i]),
        "dqmc_engine_sync": (i, [vp]),
        "dqmc_engine_errors": (C.c_uint, [vp]),
        "dqmc_engine_get_chain": (i, [vp, i, vp, vp, ip]),
        "dqmc_engine_get_acc": (i, [vp, i, ip, vp, ip, vp]),
        "dqmc_engine_get_g": (i, [vp, i, vp, vp, vp]),
        "dqmc_engine_accepts": (i, [vp, i, C.POINTER(C.c_longlong)]),
        "dqmc_engine_stream": (vp, [vp]),
        "dqmc_engine_lanes": (i, [vp]),
        "dqmc_engine_set_chains": (i, [vp, vp, vp, vp, vp, i]),
        "dqmc_engine_get_chains": (i, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "dqmc_engine_launches_per_sweep": (i, [vp, i, i]),
        "dqmc_engine_profile_sweep": (i, [vp, i, i, C.POINTER(C.c_double), i]),
        "dqmc_engine_profile_grad": (i, [vp, i, C.POINTER(C.c_double), i, vp]),
        "dqmc_engine_update_on_chip": (i, [vp]),
        "dqmc_engine_logdet_grad": (i, [vp, vp, vp]),
        "dqmc_engine_obs_grad": (i, [vp, vp, vp]),
        "dqmc_engine_set_hopping": (i, [vp] * 9),
        "dqmc_engine_check_g": (i, [vp, i]),
        "dqmc_engine_g_drift": (i, [vp, vp, vp, vp]),
        "dqmc_engine_g_drift_ue": (i, [vp, vp, vp, vp]),
        "dqmc_engine_g_drift_acc": (i, [vp, vp, vp, vp]),
        "dqmc_batch_create": (i, [vp, i, vp]),
        "dqmc_batch_sweeps": (i, [vp, i, i]),
        "dqmc_batch_stream": (vp, [vp]),
        "dqmc_batch_destroy": (None, [vp]),
        "dqmc_gpu_gemm": (i, [i, i, i, i, i, vp, vp, i, C.c_longlong, vp, i, C.c_longlong, vp,
                              vp, i, C.c_longlong, vp]),
        "dqmc_gpu_calc_eq_g": (i, [i, i, i, i, i, vp, vp, vp, vp]),
        "dqmc_gpu_calc_eq_g_noalloc": (i, [i, i, i, i, i, vp, vp, vp, vp]),
        "dqmc_gpu_update_delayed": (i, [i, i, i, i, vp, vp, vp, vp, vp, vp]),
        "dqmc_gpu_mul_seq": (i, [i, i, i, i, i, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _ = u64p
    _lib = lib
    return lib


def check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")
