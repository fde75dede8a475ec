"""ctypes binding of libpyfacc_b200.so (declarations: include/pyfacc_b200.h).

The library is built in-tree by ``pyfacc-scf_b200/build.py``.  There is no
fallback: if the shared object is missing or fails to load, every entry
point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.environ.get("PYFACC_LIB", os.path.join(PKG_ROOT, "lib", "libpyfacc_b200.so"))
DATA_DIR = os.path.join(PKG_ROOT, "data")

c_int, c_double, c_char_p, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_void_p
P_double = ctypes.POINTER(ctypes.c_double)
P_int32 = ctypes.POINTER(ctypes.c_int32)

OK = 0
ERR_BASIS_NOT_FOUND = 1
ERR_UNSUPPORTED_L = 2
ERR_NOT_CONVERGED = 3
ERR_LINDEP = 4
ERR_CUDA = 5
ERR_TIMEOUT = 6
ERR_INVALID = 7
ERR_ELEMENT = 8
ERR_NO_DEVICE = 9
ERR_NOT_READY = 10

BOYS_ACCURATE = 0
BOYS_REFERENCE_TRAPEZOID = 1
PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_FP32 = 2
SCF_AUTO, SCF_RHF, SCF_UHF = 0, 1, 2
GUESS_CORE, GUESS_ATOMIC = 0, 1


class Options(ctypes.Structure):
    _fields_ = [
        ("eps_energy", c_double), ("eps_diis", c_double), ("eps_density", c_double),
        ("max_iter", c_int), ("diis_size", c_int), ("scf_type", c_int), ("precision", c_int),
        ("boys_mode", c_int), ("schwarz_thresh", c_double), ("fp32_thresh", c_double),
        ("incremental", c_int), ("rebuild_every", c_int), ("compute_gradient", c_int),
        ("device", c_int), ("verbose", c_int), ("shard_rank", c_int), ("shard_count", c_int),
        ("data_dir", c_char_p), ("guess", c_int), ("incremental_thresh", c_double), ("task_width", c_int),
        ("gradient_precision", c_int), ("polish", c_int), ("gradient_fp32_thresh", c_double),
        ("coarse_err", c_double),
    ]


class MoleculeC(ctypes.Structure):
    _fields_ = [
        ("natoms", c_int), ("z", P_int32), ("coords", P_double), ("species", c_void_p),
        ("charge", c_int), ("nalpha", c_int), ("nbeta", c_int), ("basis", c_char_p),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("energy", c_double), ("e_elec", c_double), ("e_nuc", c_double),
        ("converged", c_int), ("n_iter", c_int), ("scf_type", c_int), ("nbf", c_int), ("nshell", c_int),
        ("n_fock_builds", c_int),
        ("last_delta_e", c_double), ("last_diis_error", c_double),
        ("gradient", P_double), ("S", P_double), ("T", P_double), ("V", P_double), ("P", P_double),
        ("C_alpha", P_double), ("C_beta", P_double), ("eps_alpha", P_double), ("eps_beta", P_double),
        ("ms_total", c_double), ("ms_one_electron", c_double), ("ms_fock", c_double), ("ms_diag", c_double),
        ("ms_gradient", c_double),
        ("quartets_fp64", ctypes.c_longlong), ("quartets_fp32", ctypes.c_longlong),
        ("flops_fock", c_double), ("flops_gradient", c_double), ("task_width", c_int),
    ]


REDUCE_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_void_p, ctypes.c_longlong)

# Every symbol include/pyfacc_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "run_scf_c": (None, [c_int, c_int, c_int, c_int, c_int, c_void_p, P_double, c_double, c_int, P_double,
                         c_char_p, P_int32]),
    "run_scf_interface_py": (None, [P_int32, P_int32, P_int32, P_int32, P_int32, c_void_p, P_double, P_double,
                                    P_int32, P_double, c_char_p, P_int32, P_int32]),
    "libint_overlap_c": (None, [c_int, c_int, P_double, P_double, P_double, c_int, c_int, P_double, P_double,
                                P_double, P_double]),
    "libint_kinetic_c": (None, [c_int, c_int, P_double, P_double, P_double, c_int, c_int, P_double, P_double,
                                P_double, P_double]),
    "libint_potential_c": (None, [c_int, c_int, P_double, P_double, P_double, c_int, c_int, P_double, P_double,
                                  P_double, P_double, P_double]),
    "pyfacc_last_status": (c_int, []),
    "pyfacc_status_string": (c_char_p, [c_int]),
    "pyfacc_last_message": (c_char_p, []),
    "pyfacc_default_options": (None, [ctypes.POINTER(Options)]),
    "pyfacc_run": (c_int, [ctypes.POINTER(MoleculeC), ctypes.POINTER(Options), ctypes.POINTER(Result)]),
    "pyfacc_run_batch": (c_int, [c_int, ctypes.POINTER(MoleculeC), ctypes.POINTER(Options), ctypes.POINTER(Result)]),
    "pyfacc_batch_last_stats": (c_int, [P_double, c_int]),
    "pyfacc_system_create": (c_int, [ctypes.POINTER(MoleculeC), ctypes.POINTER(Options), ctypes.POINTER(c_void_p)]),
    "pyfacc_system_destroy": (None, [c_void_p]),
    "pyfacc_system_info": (c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                   ctypes.POINTER(c_int)]),
    "pyfacc_system_set_coords": (c_int, [c_void_p, P_double]),
    "pyfacc_system_one_electron": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "pyfacc_system_jk": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int]),
    "pyfacc_system_eri_tensor": (c_int, [c_void_p, c_void_p]),
    "pyfacc_system_jk_stats": (c_int, [c_void_p, P_double, c_int]),
    "pyfacc_system_scf": (c_int, [c_void_p, ctypes.POINTER(Result)]),
    "pyfacc_system_gradient": (c_int, [c_void_p, P_double]),
    "pyfacc_system_density_dev": (c_int, [c_void_p, ctypes.POINTER(c_void_p)]),
    "pyfacc_system_result": (c_int, [c_void_p, ctypes.POINTER(Result)]),
    "pyfacc_launch_count": (ctypes.c_longlong, []),
    "pyfacc_boys_dev": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "pyfacc_partition": (c_int, [c_int, P_double, c_int, ctypes.POINTER(c_int)]),
    "pyfacc_dense_gemm_dev": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int]),
    "pyfacc_purify_dev": (c_int, [c_int, c_int, c_void_p, c_void_p, ctypes.POINTER(c_int)]),
    "pyfacc_system_set_reducer": (c_int, [c_void_p, REDUCE_FN, c_void_p]),
    "pyfacc_probe_fp64_gflops": (c_double, [c_int, P_double]),
    "pyfacc_version": (c_char_p, []),
    "pyfacc_jk_noalloc": (c_int, [ctypes.POINTER(MoleculeC), c_char_p, c_double, c_void_p, c_void_p, c_void_p]),
}

_lib = None


def lib():
    """Load the engine (raises if it is not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libpyfacc_b200.so not found at {LIB_PATH}; run pyfacc-scf_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class PyfaccError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        L = lib()
        msg = L.pyfacc_status_string(status).decode()
        detail = L.pyfacc_last_message().decode()
        super().__init__(f"{where}: {msg} (status {status}){': ' + detail if detail else ''}")
        self.status = status


def check(status: int, where: str = "", allow=(OK,)):
    if status not in allow:
        raise PyfaccError(status, where)
    return status


def default_options(**kw) -> Options:
    o = Options()
    lib().pyfacc_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if k == "data_dir":
            v = v.encode() if isinstance(v, str) else v
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k!r}")
        setattr(o, k, v)
    if o.data_dir is None:
        o.data_dir = DATA_DIR.encode()
    return o
