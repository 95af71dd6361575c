"""ctypes bindings for ``libgnomon_gpu.so`` (the C ABI in ``include/gnomon_gpu.h``).

The shared library is the product; this module only declares its signatures.
There is no fallback: if the library is missing the import of any scoring
entry point raises, naming the build step.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgnomon_gpu.so"

GNM_OK, GNM_DECLINED, GNM_ERR_IO, GNM_ERR_COMPUTE, GNM_ERR_PRODUCER, GNM_ERR_TIMEOUT, GNM_ERR_INVALID = range(7)
STATUS_NAMES = {0: "GNM_OK", 1: "GNM_DECLINED", 2: "GNM_ERR_IO", 3: "GNM_ERR_COMPUTE",
                4: "GNM_ERR_PRODUCER", 5: "GNM_ERR_TIMEOUT", 6: "GNM_ERR_INVALID"}
ENGINE_AUTO, ENGINE_PLAIN, ENGINE_TENSOR = 0, 1, 2
DEVICE_CURRENT, DEVICE_BEST = -1, -2   # device arguments besides an ordinal
# plain accumulate kernels (gnm_plan_tuned_shape >> 16): tile bytes, +1 = producer warp
PLAIN_KERNELS = (1024, 512, 513, 1025, 2049)

u8p = C.POINTER(C.c_uint8)


class gnm_error(C.Structure):
    _fields_ = [("message", C.c_char * 512)]


class gnm_prep_view(C.Structure):
    _fields_ = [
        ("num_people", C.c_uint64),
        ("total_people_in_fam", C.c_uint64),
        ("bytes_per_variant", C.c_uint64),
        ("num_scores", C.c_uint64),
        ("num_variants", C.c_uint64),
        ("sparse_weights", C.c_void_p),
        ("sparse_missing_corrections", C.c_void_p),
        ("sparse_score_columns", C.c_void_p),
        ("sparse_row_offsets", C.c_void_p),
        ("required_bim_indices", C.c_void_p),
        ("output_idx_to_fam_idx", C.c_void_p),
        ("baseline", C.c_void_p),
    ]


READ_AT = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64)
BLOCK_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p)


class gnm_bed_view(C.Structure):
    _fields_ = [("data", C.c_void_p), ("data_len", C.c_uint64), ("read_at", READ_AT),
                ("user_ctx", C.c_void_p)]


class gnm_resume(C.Structure):
    _fields_ = [("completed_variants", C.c_uint64), ("sums", C.c_void_p), ("counts", C.c_void_p)]


class gnm_run_options(C.Structure):
    _fields_ = [("engine", C.c_int), ("device", C.c_int), ("block_variants", C.c_uint64),
                ("on_block", BLOCK_CB), ("on_block_ctx", C.c_void_p)]


# name -> (restype, argtypes); every symbol include/gnomon_gpu.h declares.
SIGNATURES = {
    "gnm_abi_version": (C.c_int, []),
    "gnm_score_run": (C.c_int, [C.POINTER(gnm_prep_view), C.POINTER(gnm_bed_view),
                                C.POINTER(gnm_resume), C.c_void_p, C.c_void_p,
                                C.POINTER(gnm_error)]),
    "gnm_score_run_ex": (C.c_int, [C.POINTER(gnm_prep_view), C.POINTER(gnm_bed_view),
                                   C.POINTER(gnm_resume), C.POINTER(gnm_run_options),
                                   C.c_void_p, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_plan_create": (C.c_int, [C.POINTER(gnm_prep_view), C.c_int, C.c_int,
                                  C.POINTER(C.c_void_p), C.POINTER(gnm_error)]),
    "gnm_plan_destroy": (None, [C.c_void_p]),
    "gnm_plan_engine": (C.c_int, [C.c_void_p]),
    "gnm_plan_device_bytes": (C.c_uint64, [C.c_void_p]),
    "gnm_plan_reset": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_plan_accumulate_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64,
                                             C.c_uint64, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_plan_finalize_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.POINTER(gnm_error)]),
    "gnm_plan_sync": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_score_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_plan_launch_count": (C.c_uint64, [C.c_void_p]),
    "gnm_plan_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p,
                                    C.POINTER(gnm_error)]),
    "gnm_plan_tuned_shape": (C.c_uint32, [C.c_void_p]),
    "gnm_plan_set_shape": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(gnm_error)]),
    "gnm_plan_set_backward_limbs": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(gnm_error)]),
    "gnm_decode_device": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                    C.c_uint64, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_release_cached_memory": (C.c_int, [C.c_int, C.POINTER(gnm_error)]),
    "gnm_watchdog_selftest": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_uint64),
                                        C.POINTER(gnm_error)]),
    "gnm_synth_fill_device": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64,
                                        C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
                                        C.POINTER(gnm_error)]),
    "gnm_backward_dw_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(gnm_error)]),
    "gnm_pgen_dims": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                                C.POINTER(C.c_uint64), C.POINTER(gnm_error)]),
    "gnm_pgen_decode_device": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.c_void_p, C.c_uint64,
                                         C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_pgen_open": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(C.c_void_p),
                                C.POINTER(gnm_error)]),
    "gnm_pgen_close": (None, [C.c_void_p]),
    "gnm_pgen_device_bytes": (C.c_uint64, [C.c_void_p]),
    "gnm_pgen_decode": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64,
                                  C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_pgen_check": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_pgen_decode_list": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                       C.c_uint64, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_pgen_open_alleles": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_void_p), C.POINTER(gnm_error)]),
    "gnm_pgen_decode_alleles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                          C.c_void_p, C.c_uint64, C.c_void_p,
                                          C.POINTER(gnm_error)]),
    "gnm_score_pgen_alleles": (C.c_int, [C.POINTER(gnm_prep_view), C.c_void_p, C.c_uint64,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                         C.POINTER(gnm_run_options), C.c_void_p, C.c_void_p,
                                         C.POINTER(gnm_error)]),
    "gnm_project_create": (C.c_int, [C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_void_p),
                                     C.POINTER(gnm_error)]),
    "gnm_project_destroy": (None, [C.c_void_p]),
    "gnm_project_block": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                    C.POINTER(gnm_error)]),
    "gnm_project_scores": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(gnm_error)]),
    "gnm_score_pgen": (C.c_int, [C.POINTER(gnm_prep_view), C.c_void_p, C.c_uint64,
                                 C.POINTER(gnm_run_options), C.c_void_p, C.c_void_p,
                                 C.POINTER(gnm_error)]),
    "gnm_score_noalloc": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.POINTER(gnm_error)]),
}

_LIB = None


class GnomonGpuError(RuntimeError):
    """A non-OK gnm_status; ``status`` holds the code, the message the reason."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load() -> C.CDLL:
    """Load the library (once).  Raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m gnomon_b200.build` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(status: int, err: gnm_error) -> None:
    if status != GNM_OK:
        raise GnomonGpuError(status, err.message.decode(errors="replace"))
