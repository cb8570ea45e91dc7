"""ctypes binding of libferray_b200.so (include/ferray_gpu.h).

Loading fails loudly when the shared library is missing: there is no CPU
fallback anywhere in this package.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libferray_b200.so")

# fg_status
FG_OK = 0
FG_ERR_SHAPE = 1
FG_ERR_DTYPE = 2
FG_ERR_OOM = 3
FG_ERR_BUDGET = 4
FG_ERR_TIMEOUT = 5
FG_ERR_DEVICE = 6
FG_ERR_INVALID = 7
FG_ERR_UNSUPPORTED = 8
FG_ERR_BROADCAST = 9

# fg_dtype
FG_F64, FG_F32, FG_C64, FG_C32, FG_I8, FG_U8I8, FG_I16, FG_BF16, FG_F16 = range(9)
# fg_mode
FG_MODE_PLAIN, FG_MODE_SPLIT, FG_MODE_SPLIT_F16 = 0, 1, 2
FG_SHARD_LPT, FG_SHARD_ONLINE = 0, 1
FG_PROBE_INT8, FG_PROBE_BF16, FG_PROBE_FP64, FG_PROBE_FFMA = 0, 1, 2, 3


class fg_problem(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("k", C.c_int64),
                ("a", C.c_void_p), ("b", C.c_void_p), ("c", C.c_void_p),
                ("lda", C.c_int64), ("ldb", C.c_int64), ("ldc", C.c_int64)]


class fg_request(C.Structure):
    _fields_ = [("dtype", C.c_int), ("mode", C.c_int), ("m", C.c_int64), ("n", C.c_int64),
                ("k", C.c_int64), ("a", C.c_void_p), ("b", C.c_void_p), ("c", C.c_void_p),
                ("scratch_bytes", C.c_size_t)]


class fg_server_stats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("launches", C.c_uint64),
                ("grouped_launches", C.c_uint64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("useful_flops", C.c_double),
                ("busy_seconds", C.c_double), ("hbm_in_use", C.c_size_t),
                ("hbm_peak", C.c_size_t)]


class fg_profile_entry(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_uint64), ("total_ms", C.c_double)]


# Every exported symbol with (restype, argtypes); also the list the
# "library exports every declared symbol" test checks against the header.
_p, _sz, _i, _i64, _u64, _d, _f = (C.c_void_p, C.c_size_t, C.c_int, C.c_int64, C.c_uint64,
                                   C.c_double, C.c_float)
SIGNATURES = {
    "fg_init": (_i, [_i, C.POINTER(_p)]),
    "fg_shutdown": (_i, [_p]),
    "fg_sync": (_i, [_p, _p]),
    "fg_status_string": (C.c_char_p, [_i]),
    "fg_last_error": (C.c_char_p, []),
    "fg_launch_count": (_u64, []),
    "fg_profile_enable": (_i, [_i]),
    "fg_profile_collect": (_i, [C.POINTER(fg_profile_entry), _i, C.POINTER(_i)]),
    "fg_device_info": (_i, [_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_sz)]),
    "fg_selftest_wait_timeout": (_i, [_p, C.c_uint32, _p]),
    "fg_npy_parse": (_i, [_p, _sz, C.POINTER(_i), C.POINTER(_i64), C.POINTER(_i), C.POINTER(_i),
                          C.POINTER(_sz)]),
    "fg_npy_upload": (_i, [_p, _p, _sz, C.POINTER(_p), C.POINTER(_i), C.POINTER(_i64), C.POINTER(_i), _p]),
    "fg_npz_count": (_i, [_p, _sz, C.POINTER(_sz)]),
    "fg_npz_name": (_i, [_p, _sz, _sz, C.c_char_p, _sz, C.POINTER(_sz)]),
    "fg_npz_read": (_i, [_p, _sz, C.c_char_p, _p, _sz, C.POINTER(_sz)]),
    "fg_npz_upload": (_i, [_p, _p, _sz, C.c_char_p, C.POINTER(_p), C.POINTER(_i), C.POINTER(_i64),
                           C.POINTER(_i), _p]),
    "fg_multi_dot": (_i, [_p, _i, _i, _sz, C.POINTER(_p), C.POINTER(_i64), _p, _p]),
    "fg_multi_dot_order": (_i, [_sz, C.POINTER(_i64), C.POINTER(_sz)]),
    "fg_matrix_power": (_i, [_p, _i, _i, _sz, _p, _i64, _p, _p]),
    "fg_trsm_left": (_i, [_p, _i, _i, _i, _i, _sz, _sz, _p, _p, _sz, _p, _sz, _p]),
    "fg_einsum": (_i, [_p, _i, _i, C.c_char_p, _p, _i, C.POINTER(_i64), _p, _i, C.POINTER(_i64), _p,
                       C.POINTER(_i64), C.POINTER(_i), _p]),
    "fg_tensordot": (_i, [_p, _i, _i, _p, _i, C.POINTER(_i64), _p, _i, C.POINTER(_i64), _i,
                          C.POINTER(_i), C.POINTER(_i), _p, C.POINTER(_i64), C.POINTER(_i), _p]),
    "fg_tune_lookup": (_i, [_i, _sz, _sz, _sz, C.POINTER(_i), C.POINTER(_i)]),
    "fg_tune_force": (_i, [_i, _i, _i]),
    "fg_tune_variants": (_i, [_i, C.POINTER(_i)]),
    "fg_buffer_alloc": (_i, [_p, _sz, C.POINTER(_p)]),
    "fg_buffer_free": (_i, [_p, _p]),
    "fg_upload": (_i, [_p, _p, _p, _sz, _p]),
    "fg_download": (_i, [_p, _p, _p, _sz, _p]),
    "fg_host_register": (_i, [_p, _p, _sz]),
    "fg_host_unregister": (_i, [_p, _p]),
    "fg_gemm_f64": (_i, [_p, _i, _i, _sz, _sz, _sz, _d, _p, _p, _d, _p, _p]),
    "fg_gemm_f32": (_i, [_p, _i, _sz, _sz, _sz, _f, _p, _p, _f, _p, _p]),
    "fg_gemm_c64": (_i, [_p, _i, _i, _sz, _sz, _sz, _d, _d, _p, _p, _d, _d, _p, _p]),
    "fg_gemm_c32": (_i, [_p, _i, _sz, _sz, _sz, _f, _f, _p, _p, _f, _f, _p, _p]),
    "fg_gemm_i8_signed": (_i, [_p, _sz, _sz, _sz, _p, _p, _p, _i, _p]),
    "fg_gemm_i8": (_i, [_p, _sz, _sz, _sz, _p, _p, _p, _i, _p]),
    "fg_gemm_i16": (_i, [_p, _sz, _sz, _sz, _p, _p, _p, _i, _p]),
    "fg_gemm_bf16_f32": (_i, [_p, _sz, _sz, _sz, _p, _p, _p, _i, _p]),
    "fg_gemm_f16_f32": (_i, [_p, _sz, _sz, _sz, _p, _p, _p, _i, _p]),
    "fg_quantized_matmul": (_i, [_p, _sz, _sz, _sz, _p, C.c_uint8, _f, _p, C.c_int8, _f, _p,
                                 _i, _p]),
    "fg_quantized_matmul_noalloc": (_i, [_p, _sz, _sz, _sz, _p, C.c_uint8, _f, _p, C.c_int8, _f,
                                         _p, _i, _p]),
    "fg_gemm": (_i, [_p, _i, _i, _i, _sz, _sz, _sz, _p, _p, _sz, _p, _sz, _p, _p, _sz, _i, _p]),
    "fg_gemm_f64_host": (_i, [_p, _i, _i, _sz, _sz, _sz, _d, _p, _p, _d, _p]),
    "fg_gemm_f32_host": (_i, [_p, _i, _sz, _sz, _sz, _f, _p, _p, _f, _p]),
    "fg_gemm_host": (_i, [_p, _i, _i, _i, _sz, _sz, _sz, _p, _p, _p, _p, _p, _i]),
    "fg_gemm_batched_strided": (_i, [_p, _i, _i, _i, _sz, _sz, _sz, _sz, _p, _p, _sz, _i64, _p,
                                     _sz, _i64, _p, _p, _sz, _i64, _i, _p]),
    "fg_matmul": (_i, [_p, _i, _i, _p, _i, C.POINTER(_i64), _p, _i, C.POINTER(_i64), _p,
                       C.POINTER(_i64), C.POINTER(_i), _p]),
    "fg_gemm_grouped": (_i, [_p, _i, _i, C.POINTER(fg_problem), _sz, _p]),
    "fg_grouped_plan_create": (_i, [_p, _i, _i, C.POINTER(fg_problem), _sz, _p,
                                    C.POINTER(_p)]),
    "fg_grouped_plan_run": (_i, [_p, _p]),
    "fg_probe_peak": (_i, [_p, _i, C.POINTER(C.c_double)]),
    "fg_shard_plan": (_i, [_p, _p, _sz, _i, _i, _i, _p, C.POINTER(_sz)]),
    "fg_gemm_grouped_shard": (_i, [_p, _i, _i, C.POINTER(fg_problem), _sz, _i, _i, _p]),
    "fg_grouped_plan_destroy": (_i, [_p]),
    "fg_server_start": (_i, [_p, _sz, _i, _i, C.POINTER(_p)]),
    "fg_server_submit": (_i, [_p, C.POINTER(fg_request), C.POINTER(_u64)]),
    "fg_server_wait": (_i, [_p, _u64, _i64]),
    "fg_server_wait_times": (_i, [_p, _u64, _i64, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fg_server_clock": (C.c_double, []),
    "fg_server_stats_get": (_i, [_p, C.POINTER(fg_server_stats)]),
    "fg_server_stop": (_i, [_p]),
}

_lib = None


def load():
    """Load and declare the library (raises OSError when it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libferray_b200.so is not built (run ferray_b200/build.py); "
                          "this package has no CPU fallback")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
