"""ctypes binding of libbipp_b200.so (the C ABI declared in include/bipp_b200.h).

The library is loaded from this package directory; there is no fallback: if the
shared object is missing or cannot be loaded, importing raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbipp_b200.so")

BIPP_PU_AUTO, BIPP_PU_CPU, BIPP_PU_GPU = 0, 1, 2
BIPP_PRECISION_SINGLE, BIPP_PRECISION_DOUBLE = 0, 1

ERROR_NAMES = [
    "BIPP_SUCCESS", "BIPP_GENERIC_ERROR", "BIPP_INTERNAL_ERROR", "BIPP_INVALID_PARAMETER_ERROR",
    "BIPP_INVALID_POINTER_ERROR", "BIPP_INVALID_HANDLE_ERROR", "BIPP_EIGENSOLVER_ERROR",
    "BIPP_NOT_IMPLEMENTED_ERROR", "BIPP_GPU_ERROR", "BIPP_GPU_SUPPORT_ERROR", "BIPP_GPU_BLAS_ERROR",
    "BIPP_INVALID_ALLOCATOR_FUNCTION", "BIPP_MPI_ERROR", "BIPP_HDF5_ERROR", "BIPP_FILE_ERROR",
]

_sz, _p, _i, _f, _d = C.c_size_t, C.c_void_p, C.c_int, C.c_float, C.c_double
_pf, _pd, _psz = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_size_t)


class NufftOptions(C.Structure):
    _fields_ = [("precision", _i), ("tolerance", _f), ("sampleBatchSize", _sz), ("partitionMethod", _i),
                ("partitionGrid", _sz * 3), ("normalizeImage", _i), ("applyScaling", _i)]


NUM_SAMPLES_FN = C.CFUNCTYPE(_sz, _p)
EIG_VEC_FN = C.CFUNCTYPE(None, _p, _sz, _p, _sz)
EIG_VAL_FN = C.CFUNCTYPE(None, _p, _sz, _pf)
UVW_FN = C.CFUNCTYPE(None, _p, _sz, _pf, _sz)
SCALAR_FN = C.CFUNCTYPE(_f, _p, _sz)


class DatasetCallbacks(C.Structure):
    _fields_ = [("user", _p), ("num_samples", NUM_SAMPLES_FN), ("num_antenna", NUM_SAMPLES_FN),
                ("num_beam", NUM_SAMPLES_FN), ("eig_vec", EIG_VEC_FN), ("eig_val", EIG_VAL_FN),
                ("uvw", UVW_FN), ("wl", SCALAR_FN), ("scale", SCALAR_FN)]


class PipelineConfig(C.Structure):
    _fields_ = [("nAntenna", _sz), ("nLevels", _sz), ("intervals", _pd), ("filter", _i), ("tolerance", _d),
                ("gridA", _sz), ("gridB", _sz), ("lattice", _d * 6), ("pixelN", _pd), ("uvwBasis", _pd),
                ("chunkSteps", _sz), ("maxSteps", _sz), ("mode", _i), ("vvPrecision", _i)]


# symbol -> argtypes (all return BippError as int unless listed in _RESTYPE)
SIGNATURES = {
    "bipp_last_error": [],
    "bipp_kernel_launch_count": [],
    "bipp_ctx_create": [_i, C.POINTER(_p)],
    "bipp_ctx_create_on_device": [_i, _i, C.POINTER(_p)],
    "bipp_ctx_destroy": [_p],
    "bipp_ctx_processing_unit": [_p, C.POINTER(_i)],
    "bipp_ctx_stream": [_p, C.POINTER(_p)],
    "bipp_eigh_gram_s": [_p, _f, _sz, _sz, _p, _sz, _p, _sz, _p, _sz, _p, _p, _sz, _psz, _pf],
    "bipp_eigh_gram_d": [_p, _d, _sz, _sz, _p, _sz, _p, _sz, _p, _sz, _p, _p, _sz, _psz, _pd],
    "bipp_eigh_s": [_p, _f, _sz, _sz, _p, _sz, _p, _sz, _p, _p, _sz, _psz, _pf],
    "bipp_eigh_d": [_p, _d, _sz, _sz, _p, _sz, _p, _sz, _p, _p, _sz, _psz, _pd],
    "bipp_eigh_gram_batched_s": [_p, _sz, _sz, _p, _p, _p, _p, _p, _p, _p],
    "bipp_eigh_gram_batched_d": [_p, _sz, _sz, _p, _p, _p, _p, _p, _p, _p],
    "bipp_eigh_gram_batched_ranked_s": [_p, _sz, _sz, _p, _p, _p, _d, _i, _p, _i, _d, _p, _p, _p, _p, _p, _p, _p],
    "bipp_rank_features_s": [_p, _sz, _sz, _p, _p, _p, _d, _p, _p],
    "bipp_rank_mlp_num_params": [],
    "bipp_rank_mlp_forward": [_p, _p, _p, _sz, _p],
    "bipp_rank_mlp_gradient": [_p, _p, _p, _p, _sz, _p, _p],
    "bipp_rank_mlp_train": [_p, _p, _p, _p, _sz, _p, _p, _sz, _i, _f, _f, _i, _p, _p],
    "bipp_autotune_pipeline": [_p, _sz, _p, _p, _p, _i, _i, _p, _sz],
    "bipp_selftest_wait_timeout": [_p, _i, C.POINTER(_i)],
    "bipp_pipeline_stage": [_p, _sz, _p, _p, _p],
    "bipp_pipeline_process_staged": [_p],
    "bipp_tuning_get": [C.c_char_p, C.POINTER(_i)],
    "bipp_tuning_set": [C.c_char_p, _i],
    "bipp_tuning_describe": [_p, _sz],
    "bipp_tuning_save": [C.c_char_p],
    "bipp_tuning_load": [C.c_char_p],
    "bipp_tuning_reset": [],
    "bipp_eigh_gram_noalloc_s": [_i, _p, _f, _sz, _p, _sz, _p, _sz, _p, _p, _sz, _p, _p, _p],
    "bipp_gram_matrix_s": [_p, _sz, _sz, _p, _sz, _p, _sz, _f, _p, _sz],
    "bipp_gram_matrix_d": [_p, _sz, _sz, _p, _sz, _p, _sz, _d, _p, _sz],
    "bipp_virtual_vis_s": [_p, _f, _sz, _sz, _p, _p, _sz, _p],
    "bipp_virtual_vis_d": [_p, _d, _sz, _sz, _p, _p, _sz, _p],
    "bipp_nuft_sum_s": [_p, _f, _sz, _p, _p, _p, _p, _sz, _p, _p, _p, _p],
    "bipp_nuft_sum_d": [_p, _d, _sz, _p, _p, _p, _p, _sz, _p, _p, _p, _p],
    "bipp_nuft_sum_multi_device": [_p, _d, _sz, _sz, _p, _sz, _p, _p, _p, _sz, _p, _p, _p, _p, _sz, _i],
    "bipp_domain_partition_grid_s": [_p, _p, _sz, _p, _p, _p, _p, _p, _p],
    "bipp_domain_partition_grid_d": [_p, _p, _sz, _p, _p, _p, _p, _p, _p],
    "bipp_nufft_create": [_p, C.POINTER(NufftOptions), _sz, _p, _sz, _sz, _sz, C.POINTER(_p)],
    "bipp_nufft_add_s": [_p, _p, _sz, _p, _sz],
    "bipp_nufft_add_d": [_p, _p, _sz, _p, _sz],
    "bipp_nufft_get_image": [_p, _sz, _p],
    "bipp_nufft_destroy": [_p],
    "bipp_image_synthesis": [_p, C.POINTER(NufftOptions), C.POINTER(DatasetCallbacks), _sz, _sz, _p, _p, _sz, _p,
                             _sz, _p],
    "bipp_pipeline_create": [_p, C.POINTER(PipelineConfig), C.POINTER(_p)],
    "bipp_pipeline_process": [_p, _sz, _p, _p, _p, _i],
    "bipp_pipeline_images": [_p, _p, _i, _i],
    "bipp_pipeline_reset": [_p],
    "bipp_pipeline_last_eigenvalues": [_p, _p, _p],
    "bipp_pipeline_stage_times": [_p, _i, _p],
    "bipp_pipeline_kernel_times": [_p, _p],
    "bipp_pipeline_nufft_stats": [_p, _p],
    "bipp_pipeline_destroy": [_p],
}

_lib = None


RESTYPES = {"bipp_last_error": C.c_char_p, "bipp_kernel_launch_count": C.c_ulonglong}


def load(path: str = LIB_PATH):
    """Load the shared library and declare every exported entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libbipp_b200.so not found at {path}; build it with `python -m bipp_b200.build`")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = RESTYPES.get(name, C.c_int)
    _lib = lib
    return lib


class BippError(RuntimeError):
    def __init__(self, code: int, msg: str):
        name = ERROR_NAMES[code] if 0 <= code < len(ERROR_NAMES) else str(code)
        super().__init__(f"{name}: {msg}")
        self.code = code
        self.name = name


class EigensolverError(BippError):
    pass


class InvalidParameterError(BippError):
    pass


class GPUError(BippError):
    pass


_ERROR_TYPES = {6: EigensolverError, 3: InvalidParameterError, 8: GPUError, 9: GPUError}


def check(rc: int) -> None:
    if rc != 0:
        msg = load().bipp_last_error()
        msg = msg.decode() if msg else ""
        raise _ERROR_TYPES.get(rc, BippError)(rc, msg)
