"""Loads liblible_b200.so and declares the C ABI of include/lible_b200.h for ctypes."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblible_b200.so")

STATUS = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ENOSTRUCT", 4: "ENORI", 5: "EUNSUPPORTED", 6: "ETIMEOUT",
          7: "EINTERNAL"}


class LibleGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class JKOpts(ctypes.Structure):
    _fields_ = [("schwarz_threshold", ctypes.c_double), ("fp32_threshold", ctypes.c_double),
                ("precision", ctypes.c_int), ("use_graph", ctypes.c_int)]


class JKStats(ctypes.Structure):
    _fields_ = [("n_quartets", ctypes.c_longlong), ("n_fp32", ctypes.c_longlong), ("n_launches", ctypes.c_longlong)]


class JKPlanInfo(ctypes.Structure):
    _fields_ = [("n_quartets", ctypes.c_longlong), ("n_fp32", ctypes.c_longlong),
                ("n_prim_quartets", ctypes.c_longlong), ("n_launches", ctypes.c_longlong),
                ("flops_fp64", ctypes.c_double), ("flops_fp32", ctypes.c_double)]


class RIKInfo(ctypes.Structure):
    _fields_ = [("n_pos", ctypes.c_longlong), ("n_neg", ctypes.c_longlong), ("n_blocks", ctypes.c_int),
                ("t_ints", ctypes.c_double), ("t_gemm", ctypes.c_double), ("t_solve", ctypes.c_double),
                ("t_syrk", ctypes.c_double), ("flops_gemm", ctypes.c_double), ("flops_solve", ctypes.c_double),
                ("flops_syrk", ctypes.c_double), ("fitted", ctypes.c_int)]


# name -> argument types; every function returns int (status) unless noted
P = ctypes.c_void_p
I = ctypes.c_int
LL = ctypes.c_longlong
D = ctypes.c_double
S = ctypes.c_char_p
SIGNATURES = {
    "lible_gpu_create": [I, ctypes.POINTER(P)],
    "lible_gpu_destroy": [P],
    "lible_gpu_set_structure_named": [P, S, S, S, S, I, P, P, I],
    "lible_gpu_set_structure": [P, I, P, P, I, P, P, P, P, P, P, P, P, P, P],
    "lible_gpu_dims": [P, P, P, P, P],
    "lible_gpu_eri4": [P, P],
    "lible_gpu_eri4_diagonal": [P, P],
    "lible_gpu_eri3": [P, P],
    "lible_gpu_eri2": [P, P],
    "lible_gpu_eri2_diagonal": [P, P],
    "lible_gpu_pair_classes": [P, I, P, P, P, P],
    "lible_gpu_aux_classes": [P, P, P, P],
    "lible_gpu_eri4_batch": [P, I, I, I, LL, P, P],
    "lible_gpu_eri4d1_batch": [P, I, I, I, LL, P, P],
    "lible_gpu_eri4_batch_noalloc": [P, I, I, I, LL, P, P],
    "lible_gpu_eri3_batch": [P, I, I, I, LL, P, P],
    "lible_gpu_eri3d1_batch": [P, I, I, I, LL, P, P],
    "lible_gpu_eri2_batch": [P, I, I, LL, P, P],
    "lible_gpu_eri2d1_batch": [P, I, I, LL, P, P],
    "lible_gpu_eri4soc_batch": [P, I, I, I, LL, P, P],
    "lible_gpu_eri3soc_batch": [P, I, I, I, LL, P, P],
    "lible_gpu_eri2d2_batch": [P, I, I, LL, P, P],
    "lible_gpu_jk": [P, P, P, P, ctypes.POINTER(JKOpts), ctypes.POINTER(JKStats)],
    "lible_gpu_jk_energy_forward": [P, P, ctypes.POINTER(JKOpts), P, P, P],
    "lible_gpu_jk_energy_backward": [P, P, ctypes.POINTER(JKOpts), P],
    "lible_gpu_rij": [P, P, D, P, P, P],
    "lible_gpu_jk_plan": [P, ctypes.POINTER(JKOpts), ctypes.POINTER(JKPlanInfo)],
    "lible_gpu_set_batch": [P, I, S, P, P, P, P, I],
    "lible_gpu_batch_layout": [P, P, P, P, P],
    "lible_gpu_jk_autotune": [P, P, P, P, ctypes.POINTER(JKOpts), S, P, I],
    "lible_gpu_set_tune_cache": [P, S],
    "lible_gpu_jk_profile": [P, P, P, P, ctypes.POINTER(JKOpts), P, P, P, P, P, P],
    "lible_gpu_stream": [P, ctypes.POINTER(P)],
    "lible_gpu_jk_plan_classes": [P, ctypes.POINTER(JKOpts), P, P, P, P, P, P],
    "lible_gpu_fp64_peak": [P, ctypes.POINTER(D), ctypes.POINTER(D)],
    "lible_gpu_fp32_peak": [P, ctypes.POINTER(D), ctypes.POINTER(D)],
    "lible_gpu_check_bounded_wait": [P, ctypes.c_int],
    "lible_gpu_inject_wait_timeout": [P, ctypes.c_int],
    "lible_gpu_eval_special": [P, ctypes.c_int, ctypes.c_int, LL, P, P],
    "lible_gpu_ri_contract": [P, P, P, D, P, P],
    "lible_gpu_rij_last_solve": [P, P, P, P, P, P],
    "lible_gpu_rik": [P, P, P, LL, D, P, ctypes.POINTER(RIKInfo)],
    "lible_gpu_rik_set_fitted": [P, I],
    "lible_gpu_rij_set_cached": [P, I],
    "lible_gpu_rij_grad": [P, P, D, P, ctypes.POINTER(D)],
    "lible_gpu_overlap": [P, P],
    "lible_gpu_kinetic_energy": [P, P],
    "lible_gpu_nuclear_attraction": [P, P],
    "lible_gpu_external_charges": [P, P, I, P],
    "lible_gpu_one_electron": [P, P, I, P, P, P],
    "lible_gpu_one_electron_batch": [P, I, I, I, LL, P, P, I, P],
    "lible_gpu_one_electron_batch_ex": [P, I, I, I, LL, P, P, P, I, P, P],
    "lible_gpu_dipole_moment": [P, P, P],
    "lible_gpu_momentum": [P, P],
    "lible_gpu_angular_momentum": [P, P, P],
    "lible_gpu_nuclear_attraction_erf": [P, P, P],
    "lible_gpu_spin_orbit_coupling_1el": [P, P],
    "lible_gpu_pvp_integrals": [P, P, I, P],
    "lible_gpu_external_charges_erf": [P, P, P, I, P],
    "lible_gpu_one_electron_grad": [P, P, P, P],
    "lible_host_spherical_trafo": [I, P, P, P, P],
    "lible_host_shell_norms": [I, I, P, P, P],
    "lible_host_pair_classes": [S, S, I, P, P, I, I, P, P, P, P],
    "lible_host_boys": [I, D, P],
}

_lib = None


def load():
    """Returns the loaded library; raises if the CUDA extension has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m lible_b200.build` "
                           "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.lible_gpu_last_error.argtypes = [P]
    lib.lible_gpu_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def check(ctx, code):
    if code != 0:
        msg = load().lible_gpu_last_error(ctx)
        raise LibleGpuError(code, msg.decode() if msg else "")
