"""ctypes binding of libpm3gpu.so (the C ABI declared in include/pm3gpu.h)."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpm3gpu.so")

OK = 0
GUESS_LEARNED = 4
GUESS_PARAMS = 150280
PRECISION_FP64 = 0
PRECISION_MIXED = 1
TUNE_BATCH_TIME = 0
TUNE_THROUGHPUT = 1
INVALID_INPUT = 1
MISSING_ELEMENT = 2
RESOURCE_LIMIT = 3
SCF_NOT_CONVERGED = 4
LINALG = 5
CUDA_ERROR = 6
UNSUPPORTED = 8


class Options(ctypes.Structure):
    _fields_ = [
        ("charge", ctypes.c_double),
        ("multiplicity", ctypes.c_int),
        ("max_scf", ctypes.c_int),
        ("e_tol", ctypes.c_double),
        ("p_tol", ctypes.c_double),
        ("use_diis", ctypes.c_int),
        ("accelerator", ctypes.c_int),
        ("adiis_switch", ctypes.c_double),
        ("reference", ctypes.c_int),
        ("guess", ctypes.c_int),
        ("stability", ctypes.c_int),
        ("level_shift_ev", ctypes.c_double),
        ("damping", ctypes.c_double),
        ("scf_memory_mb", ctypes.c_int),
        ("variant", ctypes.c_int),
        ("mmok", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("nao", ctypes.c_int),
        ("n_occ", ctypes.c_int),
        ("n_beta", ctypes.c_int),
        ("electronic_ev", ctypes.c_double),
        ("core_ev", ctypes.c_double),
        ("total_ev", ctypes.c_double),
        ("heat_of_formation_kcal", ctypes.c_double),
        ("dipole_debye", ctypes.c_double * 3),
        ("dipole_magnitude", ctypes.c_double),
        ("homo_ev", ctypes.c_double),
        ("lumo_ev", ctypes.c_double),
        ("has_homo", ctypes.c_int),
        ("has_lumo", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("unrestricted", ctypes.c_int),
        ("scf_paths_tried", ctypes.c_int),
        ("scf_improvement_ev", ctypes.c_double),
        ("last_change", ctypes.c_double),
    ]


class OptOptions(ctypes.Structure):
    """pm3gpu_opt_options: OptOptions of pm3-rs src/optimizer.rs:15-35 (max_iter, gtol, history)."""
    _fields_ = [("max_iter", ctypes.c_int), ("gtol", ctypes.c_double), ("history", ctypes.c_int)]


class OptResult(ctypes.Structure):
    """pm3gpu_opt_result: one molecule's optimisation outcome."""
    _fields_ = [
        ("status", ctypes.c_int), ("converged", ctypes.c_int), ("iterations", ctypes.c_int),
        ("evaluations", ctypes.c_int), ("energy_ev", ctypes.c_double), ("heat_of_formation_kcal", ctypes.c_double),
        ("max_gradient", ctypes.c_double),
    ]


class Element(ctypes.Structure):
    """pm3gpu_element: the Pm3Element fields of the s/p path (pm3-rs src/params.rs:20-92)."""
    _fields_ = [
        ("z", ctypes.c_int), ("n_orb", ctypes.c_int), ("npq", ctypes.c_int), ("n_gauss", ctypes.c_int),
        ("u_ss", ctypes.c_double), ("u_pp", ctypes.c_double), ("zeta_s", ctypes.c_double),
        ("zeta_p", ctypes.c_double), ("beta_s", ctypes.c_double), ("beta_p", ctypes.c_double),
        ("g_ss", ctypes.c_double), ("g_sp", ctypes.c_double), ("g_pp", ctypes.c_double), ("g_p2", ctypes.c_double),
        ("h_sp", ctypes.c_double), ("alpha", ctypes.c_double), ("gauss", (ctypes.c_double * 3) * 4),
        ("core_charge", ctypes.c_double), ("occ_s", ctypes.c_double), ("occ_p", ctypes.c_double),
        ("eheat_ev", ctypes.c_double), ("e_isol", ctypes.c_double), ("mass", ctypes.c_double),
        ("dd", ctypes.c_double), ("qq", ctypes.c_double), ("rho0", ctypes.c_double), ("rho1", ctypes.c_double),
        ("rho2", ctypes.c_double), ("ddp", ctypes.c_double * 7), ("po", ctypes.c_double * 10),
    ]


class Pair(ctypes.Structure):
    """pm3gpu_pair: PairParams (pm3-rs src/params.rs:104-109)."""
    _fields_ = [("zi", ctypes.c_int), ("zj", ctypes.c_int), ("alpha", ctypes.c_double), ("x", ctypes.c_double)]


# Every symbol include/pm3gpu.h declares.
EXPORTS = [
    "pm3gpu_default_options", "pm3gpu_supported_element", "pm3gpu_result_sizes",
    "pm3gpu_context_create", "pm3gpu_context_destroy", "pm3gpu_last_error_message",
    "pm3gpu_set_stream", "pm3gpu_single_point", "pm3gpu_gradient", "pm3gpu_batch",
    "pm3gpu_batch_device_inputs", "pm3gpu_core_hamiltonian", "pm3gpu_fock", "pm3gpu_last_timings",
    "pm3gpu_last_kernel_launches", "pm3gpu_last_launch_layout", "pm3gpu_dgemm", "pm3gpu_default_opt_options",
    "pm3gpu_optimize_batch", "pm3gpu_numerical_hessian_batch", "pm3gpu_d3_batch", "pm3gpu_corrections_batch", "pm3gpu_last_transfer_bytes", "pm3gpu_last_phase_cycles",
    "pm3gpu_single_point_noalloc", "pm3gpu_set_large_threshold", "pm3gpu_last_large_phase_ms",
    "pm3gpu_set_precision", "pm3gpu_last_large_trace", "pm3gpu_autotune", "pm3gpu_load_tuning",
    "pm3gpu_tuning_choice",
    "pm3gpu_guess_train", "pm3gpu_guess_set_params", "pm3gpu_guess_get_params", "pm3gpu_guess_predict",
    "pm3gpu_standard_parameters", "pm3gpu_set_parameters", "pm3gpu_guess_gradients",
    "pm3gpu_set_large_checks", "pm3gpu_last_large_checks", "pm3gpu_split_gemm", "pm3gpu_set_tail_helpers",
    "pm3gpu_last_paired_jobs", "pm3gpu_set_tuning_goal",
]

_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int32)


def load() -> ctypes.CDLL:
    """Load the CUDA library; raises when it has not been built (there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python pm3-rs_b200/build.py` "
            "(pm3_rs runs only on the GPU library; there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.pm3gpu_default_options.argtypes = [ctypes.POINTER(Options)]
    L.pm3gpu_default_options.restype = None
    L.pm3gpu_supported_element.argtypes = [ctypes.c_int]
    L.pm3gpu_result_sizes.argtypes = [ctypes.c_int, _I, ctypes.POINTER(ctypes.c_int)]
    L.pm3gpu_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.pm3gpu_context_destroy.argtypes = [ctypes.c_void_p]
    L.pm3gpu_context_destroy.restype = None
    L.pm3gpu_last_error_message.argtypes = [ctypes.c_void_p]
    L.pm3gpu_last_error_message.restype = ctypes.c_char_p
    L.pm3gpu_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.pm3gpu_single_point.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, ctypes.POINTER(Options),
                                      ctypes.POINTER(Result), _D, _D, _D]
    L.pm3gpu_single_point_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, ctypes.POINTER(Options),
                                              ctypes.POINTER(Result), _D]
    L.pm3gpu_gradient.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, ctypes.POINTER(Options),
                                  ctypes.POINTER(Result), _D, _D]
    L.pm3gpu_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, ctypes.POINTER(Options), ctypes.c_int,
                               ctypes.POINTER(Result), _D, _D]
    L.pm3gpu_batch_device_inputs.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, _I, _I, ctypes.POINTER(Options),
                                             ctypes.POINTER(Result), _D, _D]
    L.pm3gpu_core_hamiltonian.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, _D, _D]
    L.pm3gpu_fock.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _D, _D, _D, _D, _D, _D]
    L.pm3gpu_last_timings.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
    L.pm3gpu_last_kernel_launches.argtypes = [ctypes.c_void_p]
    L.pm3gpu_default_opt_options.argtypes = [ctypes.POINTER(OptOptions)]
    L.pm3gpu_default_opt_options.restype = None
    L.pm3gpu_optimize_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, ctypes.POINTER(Options),
                                        ctypes.POINTER(OptOptions), ctypes.POINTER(OptResult), _D]
    L.pm3gpu_d3_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, ctypes.c_int, _D, _D]
    L.pm3gpu_corrections_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, ctypes.c_int, _D, _D]
    L.pm3gpu_numerical_hessian_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, ctypes.POINTER(Options),
                                                 ctypes.c_double, _D, _I]
    L.pm3gpu_dgemm.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.c_double, _D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int]
    L.pm3gpu_last_launch_layout.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.pm3gpu_set_large_threshold.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.pm3gpu_last_large_phase_ms.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
    L.pm3gpu_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.pm3gpu_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, ctypes.POINTER(Options), ctypes.c_char_p]
    L.pm3gpu_load_tuning.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    L.pm3gpu_tuning_choice.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.pm3gpu_last_large_trace.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
    L.pm3gpu_set_large_checks.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.pm3gpu_set_tail_helpers.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.pm3gpu_last_paired_jobs.argtypes = [ctypes.c_void_p]
    L.pm3gpu_set_tuning_goal.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.pm3gpu_split_gemm.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D,
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.pm3gpu_last_large_checks.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
    _F = ctypes.POINTER(ctypes.c_float)
    L.pm3gpu_guess_train.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, ctypes.POINTER(Options), ctypes.c_int,
                                     ctypes.c_int, ctypes.c_float, ctypes.c_uint, _F]
    L.pm3gpu_guess_set_params.argtypes = [ctypes.c_void_p, _F, ctypes.c_int]
    L.pm3gpu_guess_get_params.argtypes = [ctypes.c_void_p, _F, ctypes.c_int]
    L.pm3gpu_guess_predict.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _D, _F, _F]
    L.pm3gpu_guess_gradients.argtypes = [ctypes.c_void_p, ctypes.c_int, _F, _F, _F, ctypes.c_float, _F, _F]
    L.pm3gpu_last_phase_cycles.argtypes = [ctypes.c_void_p, _D, ctypes.c_int]
    L.pm3gpu_last_transfer_bytes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                             ctypes.POINTER(ctypes.c_longlong)]
    _P = ctypes.POINTER(ctypes.c_int)
    L.pm3gpu_standard_parameters.argtypes = [ctypes.POINTER(Element), ctypes.c_int, _P, ctypes.POINTER(Pair),
                                             ctypes.c_int, _P]
    L.pm3gpu_set_parameters.argtypes = [ctypes.c_void_p, ctypes.POINTER(Element), ctypes.c_int, ctypes.POINTER(Pair),
                                        ctypes.c_int]
    _lib = L
    return L


def standard_parameters():
    """Pm3Parameters::standard() of the s/p path as (elements, pairs) ctypes arrays."""
    L = load()
    ne, npair = ctypes.c_int(), ctypes.c_int()
    L.pm3gpu_standard_parameters(None, 0, ctypes.byref(ne), None, 0, ctypes.byref(npair))
    elems, pairs = (Element * ne.value)(), (Pair * npair.value)()
    rc = L.pm3gpu_standard_parameters(elems, ne.value, ctypes.byref(ne), pairs, npair.value, ctypes.byref(npair))
    if rc != OK:
        raise RuntimeError(f"pm3gpu_standard_parameters failed with status {rc}")
    return elems, pairs


class Context:
    """One CUDA device + stream + workspaces (pm3gpu_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.ptr = ctypes.c_void_p()
        rc = self.lib.pm3gpu_context_create(device, ctypes.byref(self.ptr))
        if rc != OK:
            raise RuntimeError(f"pm3gpu_context_create failed with status {rc} (is a CUDA device visible?)")

    def last_error(self) -> str:
        return self.lib.pm3gpu_last_error_message(self.ptr).decode()

    def close(self):
        if self.ptr:
            self.lib.pm3gpu_context_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = {}


def default_context(device: int = 0) -> Context:
    ctx = _default.get(device)
    if ctx is None:
        ctx = _default[device] = Context(device)
    return ctx
