"""ferray_b200 -- B200-native GEMM backend for ferray's matmul path.

Python mirror of ferray-linalg's GEMM interface over the C ABI of
libferray_b200.so (include/ferray_gpu.h).  Names, argument meaning and error
behaviour follow the reference:

* ``gemm_f64 / gemm_f32 / gemm_c64 / gemm_c32 / gemm_i8 / gemm_i8_signed /
  gemm_i16 / quantized_matmul`` keep the signatures of
  ferray-linalg/src/gemm/mod.rs (m, n, k, scalars, a, b, c[, accumulate]) and
  return ``True`` like the reference's ``-> bool`` entry points; ``False``
  means "no kernel for this case" (FG_ERR_UNSUPPORTED).
* ``matmul`` follows ferray_linalg::matmul (products/mod.rs:362-437) and
  ``matmul_complex`` (complex.rs:136-264): shape errors raise
  ``ShapeMismatch``, batch-broadcast errors ``BroadcastFailure`` -- the
  FerrayError variants of ferray-core/src/error.rs:16-99.

Operands may be host numpy arrays (staged through the device, like the
reference's slice API) or ``DeviceArray`` objects that stay resident in HBM.
Every call runs on the GPU; there is no CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _lib as L

__all__ = [
    "FerrayError", "ShapeMismatch", "BroadcastFailure", "InvalidDtype", "InvalidValue",
    "OutOfMemory", "BudgetExceeded", "DeviceTimeout", "DeviceError", "Context", "DeviceArray",
    "default_context", "gemm_f64", "gemm_f32", "gemm_c64", "gemm_c32", "gemm_i8",
    "gemm_i8_signed", "gemm_i16", "gemm_bf16_f32", "gemm_f16_f32", "quantized_matmul", "matmul", "matmul_complex",
    "gemm_batched_strided", "gemm_grouped", "GroupedPlan", "Server", "launch_count", "PLAIN",
    "SPLIT", "TUNE_OPS", "tune_lookup", "tune_forced", "multi_dot", "multi_dot_order", "matrix_power", "tensordot", "einsum",
    "trsm_left_lower_f64", "trsm_left_upper_f64", "trsm_left_lower_f32", "trsm_left_upper_f32", "npy_parse", "npy_load", "npz_names", "npz_read", "npz_load", "shard_problems",
]

PLAIN, SPLIT, SPLIT_F16 = "plain", "split", "split_f16"


class FerrayError(Exception):
    """Base class, mirrors ferray_core::FerrayError."""


class ShapeMismatch(FerrayError):
    pass


class BroadcastFailure(FerrayError):
    pass


class InvalidDtype(FerrayError):
    pass


class InvalidValue(FerrayError):
    pass


class OutOfMemory(FerrayError):
    pass


class BudgetExceeded(FerrayError):
    pass


class DeviceTimeout(FerrayError):
    pass


class DeviceError(FerrayError):
    pass


_STATUS_EXC = {
    L.FG_ERR_SHAPE: ShapeMismatch,
    L.FG_ERR_DTYPE: InvalidDtype,
    L.FG_ERR_OOM: OutOfMemory,
    L.FG_ERR_BUDGET: BudgetExceeded,
    L.FG_ERR_TIMEOUT: DeviceTimeout,
    L.FG_ERR_DEVICE: DeviceError,
    L.FG_ERR_INVALID: InvalidValue,
    L.FG_ERR_BROADCAST: BroadcastFailure,
}


class Unsupported(FerrayError):
    pass


def check(status, what=""):
    if status == L.FG_OK:
        return
    lib = L.load()
    msg = lib.fg_last_error().decode() or lib.fg_status_string(status).decode()
    exc = _STATUS_EXC.get(status, Unsupported)
    raise exc(f"{what}: {msg}" if what else msg)


def launch_count():
    """Kernels launched by libferray_b200.so in this process."""
    return int(L.load().fg_launch_count())


class Context:
    """A device context (one per GPU); thread-safe."""

    def __init__(self, device=0):
        self._lib = L.load()
        h = C.c_void_p()
        check(self._lib.fg_init(device, C.byref(h)), "fg_init")
        self.handle = h
        self.device = device

    def sync(self, stream=None):
        check(self._lib.fg_sync(self.handle, stream), "fg_sync")

    def info(self):
        sm, ma, mi, hbm = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
        check(self._lib.fg_device_info(self.handle, C.byref(sm), C.byref(ma), C.byref(mi),
                                       C.byref(hbm)))
        return {"sm_count": sm.value, "cc": (ma.value, mi.value), "hbm_bytes": hbm.value}

    def close(self):
        if getattr(self, "handle", None):
            self._lib.fg_shutdown(self.handle)
            self.handle = None


_default = None


def default_context():
    global _default
    if _default is None:
        _default = Context(0)
    return _default


_NP2FG = {np.dtype(np.float64): L.FG_F64, np.dtype(np.float32): L.FG_F32,
          np.dtype(np.complex128): L.FG_C64, np.dtype(np.complex64): L.FG_C32,
          np.dtype(np.int8): L.FG_I8, np.dtype(np.int16): L.FG_I16}
_OUT_DTYPE = {L.FG_F64: np.float64, L.FG_F32: np.float32, L.FG_C64: np.complex128,
              L.FG_C32: np.complex64, L.FG_I8: np.int32, L.FG_U8I8: np.int32,
              L.FG_I16: np.int32, L.FG_BF16: np.float32, L.FG_F16: np.float32}


def _mode(mode):
    if mode in (PLAIN, L.FG_MODE_PLAIN, None):
        return L.FG_MODE_PLAIN
    if mode in (SPLIT, L.FG_MODE_SPLIT):
        return L.FG_MODE_SPLIT
    if mode in (SPLIT_F16, L.FG_MODE_SPLIT_F16):
        return L.FG_MODE_SPLIT_F16
    raise InvalidValue(f"unknown mode {mode!r}")


class DeviceArray:
    """Row-major array resident in HBM (the device counterpart of
    ferray_core::Array, ferray-core/src/array/owned.rs:21)."""

    def __init__(self, shape, dtype, ctx=None):
        self.ctx = ctx or default_context()
        self.shape = tuple(int(s) for s in shape)
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape, dtype=np.int64)) * self.dtype.itemsize
        p = C.c_void_p()
        check(self.ctx._lib.fg_buffer_alloc(self.ctx.handle, max(self.nbytes, 1), C.byref(p)),
              "fg_buffer_alloc")
        self.ptr = p.value

    @classmethod
    def from_numpy(cls, x, ctx=None):
        x = np.ascontiguousarray(x)
        d = cls(x.shape, x.dtype, ctx)
        check(d.ctx._lib.fg_upload(d.ctx.handle, d.ptr, x.ctypes.data, x.nbytes, None), "upload")
        d.ctx.sync()
        return d

    def to_numpy(self):
        out = np.empty(self.shape, self.dtype)
        check(self.ctx._lib.fg_download(self.ctx.handle, out.ctypes.data, self.ptr, self.nbytes,
                                        None), "download")
        return out

    @property
    def ndim(self):
        return len(self.shape)

    def free(self):
        if self.ptr:
            self.ctx._lib.fg_buffer_free(self.ctx.handle, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _is_dev(x):
    return isinstance(x, DeviceArray)


def _host(x, dtype):
    return np.ascontiguousarray(x, dtype=dtype)


def _run_gemm(dtype, mode, slices, m, n, k, alpha, a, b, beta, c, accumulate, scalar_t):
    """Shared body of the gemm_* mirrors: device arrays go through the
    device entry point, host arrays through the staging entry point."""
    ctx = default_context()
    lib = ctx._lib
    al = (scalar_t * len(alpha))(*alpha)
    be = (scalar_t * len(beta))(*beta)
    if _is_dev(a) or _is_dev(b) or _is_dev(c):
        if not (_is_dev(a) and _is_dev(b) and _is_dev(c)):
            raise InvalidValue("mix of device and host operands")
        st = lib.fg_gemm(ctx.handle, dtype, _mode(mode), slices, m, n, k, al, a.ptr, k, b.ptr,
                         n, be, c.ptr, n, int(bool(accumulate)), None)
        if st == L.FG_ERR_UNSUPPORTED:
            return False
        check(st, "gemm")
        ctx.sync()
        return True
    st = lib.fg_gemm_host(ctx.handle, dtype, _mode(mode), slices, m, n, k, al,
                          a.ctypes.data, b.ctypes.data, be, c.ctypes.data, int(bool(accumulate)))
    if st == L.FG_ERR_UNSUPPORTED:
        return False
    check(st, "gemm")
    return True


def _need(x, count, dtype, name):
    if _is_dev(x):
        if x.dtype != np.dtype(dtype):
            raise InvalidDtype(f"{name}: expected {np.dtype(dtype)}, got {x.dtype}")
        if x.nbytes < count * np.dtype(dtype).itemsize:
            raise ShapeMismatch(f"{name}: buffer holds fewer than {count} elements")
        return x
    if not isinstance(x, np.ndarray) or x.dtype != np.dtype(dtype) or not x.flags.c_contiguous:
        raise InvalidDtype(f"{name}: expected a C-contiguous {np.dtype(dtype)} array")
    if x.size < count:
        raise ShapeMismatch(f"{name}: fewer than {count} elements")
    return x


def gemm_f64(m, n, k, alpha, a, b, beta, c, mode=PLAIN, ozaki_slices=0):
    """C = alpha*A@B + beta*C (gemm/mod.rs:197).  mode='split': Ozaki INT8."""
    _need(a, m * k, np.float64, "a"); _need(b, k * n, np.float64, "b")
    _need(c, m * n, np.float64, "c")
    return _run_gemm(L.FG_F64, mode, ozaki_slices, m, n, k, [alpha], a, b, [beta], c, 0,
                     C.c_double)


def gemm_f32(m, n, k, alpha, a, b, beta, c, mode=PLAIN, bf16_slices=0):
    """C = alpha*A@B + beta*C (gemm/mod.rs:940).  mode='split': 3xBF16
    (bf16_slices=2, default) or the 6-product 3-slice form (bf16_slices=3);
    mode='split_f16': 3 products of two FP16 slices of power-of-two-scaled
    operands."""
    _need(a, m * k, np.float32, "a"); _need(b, k * n, np.float32, "b")
    _need(c, m * n, np.float32, "c")
    return _run_gemm(L.FG_F32, mode, bf16_slices, m, n, k, [alpha], a, b, [beta], c, 0,
                     C.c_float)


def gemm_c64(m, n, k, alpha_re, alpha_im, a, b, beta_re, beta_im, c, mode=PLAIN,
             ozaki_slices=0):
    """Complex<f64> GEMM (gemm/mod.rs:757); a, b, c complex128."""
    _need(a, m * k, np.complex128, "a"); _need(b, k * n, np.complex128, "b")
    _need(c, m * n, np.complex128, "c")
    return _run_gemm(L.FG_C64, mode, ozaki_slices, m, n, k, [alpha_re, alpha_im], a, b,
                     [beta_re, beta_im], c, 0, C.c_double)


def gemm_c32(m, n, k, alpha_re, alpha_im, a, b, beta_re, beta_im, c, mode=PLAIN,
             bf16_slices=0):
    """Complex<f32> GEMM (gemm/mod.rs:669); a, b, c complex64."""
    _need(a, m * k, np.complex64, "a"); _need(b, k * n, np.complex64, "b")
    _need(c, m * n, np.complex64, "c")
    return _run_gemm(L.FG_C32, mode, bf16_slices, m, n, k, [alpha_re, alpha_im], a, b,
                     [beta_re, beta_im], c, 0, C.c_float)


def gemm_i8_signed(m, n, k, a, b, c, accumulate=False):
    """i8 x i8 -> i32, wrapping (gemm/mod.rs:414)."""
    _need(a, m * k, np.int8, "a"); _need(b, k * n, np.int8, "b"); _need(c, m * n, np.int32, "c")
    return _run_gemm(L.FG_I8, PLAIN, 0, m, n, k, [0.0], a, b, [0.0], c, accumulate, C.c_double)


def gemm_i8(m, n, k, a, b, c, accumulate=False):
    """u8 x i8 -> i32, exact (gemm/mod.rs:601, VNNI semantics)."""
    _need(a, m * k, np.uint8, "a"); _need(b, k * n, np.int8, "b"); _need(c, m * n, np.int32, "c")
    return _run_gemm(L.FG_U8I8, PLAIN, 0, m, n, k, [0.0], a, b, [0.0], c, accumulate,
                     C.c_double)


def gemm_i16(m, n, k, a, b, c, accumulate=False):
    """i16 x i16 -> i32, wrapping (gemm/mod.rs:348)."""
    _need(a, m * k, np.int16, "a"); _need(b, k * n, np.int16, "b"); _need(c, m * n, np.int32, "c")
    return _run_gemm(L.FG_I16, PLAIN, 0, m, n, k, [0.0], a, b, [0.0], c, accumulate,
                     C.c_double)


def gemm_bf16_f32(m, n, k, a, b, c, accumulate=False):
    """bf16 x bf16 -> f32 (gemm/mod.rs:851); a, b are uint16 arrays of bf16
    bit patterns (NumPy has no bf16 dtype), c float32."""
    _need(a, m * k, np.uint16, "a"); _need(b, k * n, np.uint16, "b"); _need(c, m * n, np.float32, "c")
    return _run_gemm(L.FG_BF16, PLAIN, 0, m, n, k, [0.0], a, b, [0.0], c, accumulate, C.c_double)


def gemm_f16_f32(m, n, k, a, b, c, accumulate=False):
    """f16 x f16 -> f32 (gemm/mod.rs:906); a, b float16 (or their uint16
    bit patterns), c float32."""
    a = a if _is_dev(a) else np.ascontiguousarray(a).view(np.uint16)
    b = b if _is_dev(b) else np.ascontiguousarray(b).view(np.uint16)
    _need(a, m * k, np.uint16 if not _is_dev(a) else a.dtype, "a")
    _need(b, k * n, np.uint16 if not _is_dev(b) else b.dtype, "b")
    _need(c, m * n, np.float32, "c")
    return _run_gemm(L.FG_F16, PLAIN, 0, m, n, k, [0.0], a, b, [0.0], c, accumulate, C.c_double)


def quantized_matmul(m, n, k, a, a_zp, scale_a, b, b_zp, scale_b, c, accumulate=False):
    """scale_a*scale_b*sum((a-a_zp)(b-b_zp)) -> f32 (gemm/mod.rs:484)."""
    _need(a, m * k, np.uint8, "a"); _need(b, k * n, np.int8, "b"); _need(c, m * n, np.float32, "c")
    ctx = default_context()
    lib = ctx._lib
    devs = [_is_dev(x) for x in (a, b, c)]
    if any(devs) and not all(devs):
        raise InvalidValue("mix of device and host operands")
    if all(devs):
        check(lib.fg_quantized_matmul(ctx.handle, m, n, k, a.ptr, a_zp, scale_a, b.ptr, b_zp,
                                      scale_b, c.ptr, int(bool(accumulate)), None), "qmm")
        ctx.sync()
        return True
    da, db, dc = (DeviceArray.from_numpy(x) for x in (a, b, c))
    check(lib.fg_quantized_matmul(ctx.handle, m, n, k, da.ptr, a_zp, scale_a, db.ptr, b_zp,
                                  scale_b, dc.ptr, int(bool(accumulate)), None), "qmm")
    ctx.sync()
    c[...] = dc.to_numpy().reshape(c.shape)
    return True


def matmul(a, b, mode=PLAIN):
    """NumPy ``@`` on the GPU (products/mod.rs:362 / complex.rs:136).

    a, b: numpy arrays or DeviceArrays of the same dtype (f64, f32, complex128,
    complex64, int8 -> int32, int16 -> int32).  Returns the same kind.
    """
    ctx = default_context()
    lib = ctx._lib
    dev = _is_dev(a)
    if dev != _is_dev(b):
        raise InvalidValue("mix of device and host operands")
    if np.dtype(a.dtype) != np.dtype(b.dtype):
        raise InvalidDtype(f"matmul: dtypes differ ({a.dtype} vs {b.dtype})")
    dt = _NP2FG.get(np.dtype(a.dtype))
    if dt is None:
        raise InvalidDtype(f"matmul: unsupported dtype {a.dtype}")
    sa = (C.c_int64 * max(len(a.shape), 1))(*a.shape)
    sb = (C.c_int64 * max(len(b.shape), 1))(*b.shape)
    os_ = (C.c_int64 * 8)()
    ond = C.c_int()
    check(lib.fg_matmul(ctx.handle, dt, _mode(mode), None, len(a.shape), sa, None, len(b.shape),
                        sb, None, os_, C.byref(ond), None), "matmul")
    out_shape = tuple(os_[i] for i in range(ond.value))
    if dev:
        da, db = a, b
    else:
        da, db = DeviceArray.from_numpy(a), DeviceArray.from_numpy(b)
    dc = DeviceArray(out_shape, _OUT_DTYPE[dt])
    check(lib.fg_matmul(ctx.handle, dt, _mode(mode), da.ptr, len(a.shape), sa, db.ptr,
                        len(b.shape), sb, dc.ptr, os_, C.byref(ond), None), "matmul")
    ctx.sync()
    return dc if dev else dc.to_numpy()


def matmul_complex(a, b, mode=PLAIN):
    """Complex 2-D matmul (complex.rs:136)."""
    if not np.issubdtype(np.dtype(a.dtype), np.complexfloating):
        raise InvalidDtype("matmul_complex: complex operands expected")
    return matmul(a, b, mode)


def gemm_batched_strided(dtype, batch, m, n, k, a, stride_a, b, stride_b, c, stride_c,
                         alpha=1.0, beta=0.0, mode=PLAIN, accumulate=False):
    """Stacked GEMM on DeviceArrays; stride 0 broadcasts an operand."""
    ctx = default_context()
    dt = _NP2FG[np.dtype(dtype)] if not isinstance(dtype, int) else dtype
    cplx = dt in (L.FG_C64, L.FG_C32)
    st_t = C.c_float if dt in (L.FG_F32, L.FG_C32) else C.c_double
    al = (st_t * 2)(complex(alpha).real, complex(alpha).imag) if cplx else (st_t * 1)(alpha)
    be = (st_t * 2)(complex(beta).real, complex(beta).imag) if cplx else (st_t * 1)(beta)
    check(ctx._lib.fg_gemm_batched_strided(ctx.handle, dt, _mode(mode), 0, batch, m, n, k, al,
                                           a.ptr, k, stride_a, b.ptr, n, stride_b, be, c.ptr, n,
                                           stride_c, int(bool(accumulate)), None), "batched")
    ctx.sync()


def _ptr(x):
    """Device address of a DeviceArray or a raw pointer (int-like or None)."""
    if _is_dev(x):
        return x.ptr
    return None if x is None else int(x)


def _table(problems):
    tab = (L.fg_problem * len(problems))()
    for i, p in enumerate(problems):
        m, n, k, a, b, c = p[:6]
        lda, ldb, ldc = p[6:9] if len(p) >= 9 else (k, n, n)
        tab[i] = L.fg_problem(m, n, k, _ptr(a), _ptr(b), _ptr(c), lda, ldb, ldc)
    return tab


def _chain_dims(arrays):
    """dims of products/mod.rs:789-815: a 1-D first operand is 1 x n, a 1-D
    last operand n x 1; every other operand must be 2-D and aligned.  (The
    reference pushes a trailing vector's length twice, so its cost model sees
    that vector as n x n; the product is the same, here the true n x 1 is
    used.)"""
    n = len(arrays)
    dims = []
    for i, x in enumerate(arrays):
        sh = x.shape
        if len(sh) != 2:
            if i == 0 and len(sh) == 1:
                dims += [1, sh[0]]
                continue
            if i == n - 1 and len(sh) == 1:
                dims.append(1)
                continue
            raise ShapeMismatch(f"multi_dot: matrix {i} has {len(sh)} dimensions (expected 2)")
        if i == 0:
            dims.append(sh[0])
        dims.append(sh[1])
    for i in range(1, n):
        prev, cur = arrays[i - 1].shape, arrays[i].shape
        if prev[-1] != cur[0]:
            raise ShapeMismatch(f"multi_dot: shapes of matrices {i - 1} and {i} not aligned "
                                f"({prev[-1]} != {cur[0]})")
    return dims


_FG2NP = {L.FG_F64: np.float64, L.FG_F32: np.float32, L.FG_C64: np.complex128, L.FG_C32: np.complex64,
          L.FG_I8: np.int8, L.FG_U8I8: np.uint8, L.FG_I16: np.int16, L.FG_F16: np.float16}


def npy_parse(data):
    """Header of an .npy byte image: (numpy dtype, shape, fortran_order,
    payload offset); host only."""
    buf = bytes(data)
    dt, nd, fo, off = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
    sh = (C.c_int64 * 8)()
    check(L.load().fg_npy_parse(buf, len(buf), C.byref(dt), sh, C.byref(nd), C.byref(fo), C.byref(off)),
          "npy_parse")
    return np.dtype(_FG2NP[dt.value]), tuple(sh[:nd.value]), bool(fo.value), off.value


def npy_load(data, ctx=None):
    """A DeviceArray holding the payload of an .npy byte image (C order)."""
    ctx = ctx or default_context()
    buf = bytes(data)
    p, dt, nd = C.c_void_p(), C.c_int(), C.c_int()
    sh = (C.c_int64 * 8)()
    check(ctx._lib.fg_npy_upload(ctx.handle, buf, len(buf), C.byref(p), C.byref(dt), sh, C.byref(nd), None),
          "npy_load")
    ctx.sync()
    arr = DeviceArray.__new__(DeviceArray)
    arr.ctx, arr.shape, arr.dtype = ctx, tuple(sh[:nd.value]), np.dtype(_FG2NP[dt.value])
    arr.nbytes = int(np.prod(arr.shape, dtype=np.int64)) * arr.dtype.itemsize
    arr.ptr = p.value
    return arr


def npz_names(data):
    """Names of the arrays in an .npz byte image, in archive order
    (NpzFile::names, ferray-io/src/npz/mod.rs:140); host only."""
    buf = bytes(data)
    lib = L.load()
    cnt = C.c_size_t()
    check(lib.fg_npz_count(buf, len(buf), C.byref(cnt)), "npz_names")
    names = []
    for i in range(cnt.value):
        n = C.c_size_t()
        check(lib.fg_npz_name(buf, len(buf), i, None, 0, C.byref(n)), "npz_names")
        out = C.create_string_buffer(n.value + 1)
        check(lib.fg_npz_name(buf, len(buf), i, out, n.value + 1, C.byref(n)), "npz_names")
        names.append(out.value.decode())
    return names


def npz_read(data, name):
    """The .npy bytes of one array of an .npz byte image (inflated, CRC
    checked); host only."""
    buf = bytes(data)
    lib = L.load()
    n = C.c_size_t()
    check(lib.fg_npz_read(buf, len(buf), name.encode(), None, 0, C.byref(n)), "npz_read")
    out = C.create_string_buffer(max(n.value, 1))
    check(lib.fg_npz_read(buf, len(buf), name.encode(), out, n.value, C.byref(n)), "npz_read")
    return out.raw[:n.value]


def npz_load(data, name, ctx=None):
    """One array of an .npz byte image as a DeviceArray (NpzFile::get,
    ferray-io/src/npz/mod.rs:150)."""
    ctx = ctx or default_context()
    buf = bytes(data)
    p, dt, nd = C.c_void_p(), C.c_int(), C.c_int()
    sh = (C.c_int64 * 8)()
    check(ctx._lib.fg_npz_upload(ctx.handle, buf, len(buf), name.encode(), C.byref(p), C.byref(dt), sh,
                                 C.byref(nd), None), "npz_load")
    ctx.sync()
    arr = DeviceArray.__new__(DeviceArray)
    arr.ctx, arr.shape, arr.dtype = ctx, tuple(sh[:nd.value]), np.dtype(_FG2NP[dt.value])
    arr.nbytes = int(np.prod(arr.shape, dtype=np.int64)) * arr.dtype.itemsize
    arr.ptr = p.value
    return arr


def multi_dot(arrays, mode=PLAIN):
    """Chain product of DeviceArrays in the reference's optimal order
    (products/mod.rs:776); intermediates stay on the device."""
    if len(arrays) < 2:
        raise InvalidValue("multi_dot: need at least 2 matrices")
    if len(arrays) == 2:
        return matmul(arrays[0], arrays[1], mode)
    dt = arrays[0].dtype
    if any(x.dtype != dt for x in arrays):
        raise InvalidDtype("multi_dot: all operands need the same dtype")
    dims = _chain_dims(arrays)
    n = len(arrays)
    shape = [dims[0], dims[-1]]
    if len(arrays[0].shape) == 1:
        shape = shape[1:]
    if len(arrays[-1].shape) == 1:
        shape = shape[:-1]
    ctx = arrays[0].ctx
    out = DeviceArray(shape, dt, ctx)
    mats = (C.c_void_p * n)(*[x.ptr for x in arrays])
    cd = (C.c_int64 * (n + 1))(*dims)
    check(ctx._lib.fg_multi_dot(ctx.handle, _NP2FG[np.dtype(dt)], _mode(mode), n, mats, cd, out.ptr, None),
          "multi_dot")
    ctx.sync()
    return out


def multi_dot_order(dims):
    """The split table fg_multi_dot uses, as a (count x count) int array."""
    n = len(dims) - 1
    cd = (C.c_int64 * (n + 1))(*dims)
    sp = (C.c_size_t * (n * n))()
    check(L.load().fg_multi_dot_order(n, cd, sp), "multi_dot_order")
    return np.array(sp[:], dtype=np.int64).reshape(n, n)


def tensordot(a, b, axes=2, mode=PLAIN):
    """numpy.tensordot on DeviceArrays (products/tensordot.rs:35): `axes` an
    int N (last N of a with first N of b) or a pair of axis lists."""
    if isinstance(axes, int):
        if axes > a.ndim or axes > b.ndim:
            raise ShapeMismatch(f"tensordot: cannot contract {axes} axes from shapes {a.shape} and {b.shape}")
        ax_a, ax_b = list(range(a.ndim - axes, a.ndim)), list(range(axes))
    else:
        ax_a, ax_b = [list(x) for x in axes]
        if len(ax_a) != len(ax_b):
            raise ShapeMismatch("tensordot: axes_a and axes_b must have the same length")
    if a.dtype != b.dtype:
        raise InvalidDtype("tensordot: operands need the same dtype")
    free_a = [a.shape[i] for i in range(a.ndim) if i not in ax_a]
    free_b = [b.shape[i] for i in range(b.ndim) if i not in ax_b]
    out = DeviceArray(free_a + free_b, a.dtype, a.ctx)
    sa = (C.c_int64 * max(a.ndim, 1))(*a.shape)
    sb = (C.c_int64 * max(b.ndim, 1))(*b.shape)
    n = len(ax_a)
    xa = (C.c_int * max(n, 1))(*ax_a)
    xb = (C.c_int * max(n, 1))(*ax_b)
    osh = (C.c_int64 * 16)()
    ond = C.c_int()
    check(a.ctx._lib.fg_tensordot(a.ctx.handle, _NP2FG[a.dtype], _mode(mode), a.ptr, a.ndim, sa, b.ptr, b.ndim,
                                  sb, n, xa, xb, out.ptr, osh, C.byref(ond), None), "tensordot")
    a.ctx.sync()
    return out


def einsum(subscripts, a, b, mode=PLAIN):
    """Two-operand einsum on DeviceArrays (pairwise contractions; see
    fg_einsum)."""
    if a.dtype != b.dtype:
        raise InvalidDtype("einsum: operands need the same dtype")
    sa = (C.c_int64 * max(a.ndim, 1))(*a.shape)
    sb = (C.c_int64 * max(b.ndim, 1))(*b.shape)
    osh = (C.c_int64 * 8)()
    ond = C.c_int()
    lib = a.ctx._lib
    # shape pass (null operands, nothing launched): the output shape
    st = lib.fg_einsum(a.ctx.handle, _NP2FG[a.dtype], _mode(mode), subscripts.encode(), None, a.ndim, sa, None,
                       b.ndim, sb, None, osh, C.byref(ond), None)
    if st not in (L.FG_OK, L.FG_ERR_INVALID):
        check(st, "einsum")
    shape = tuple(osh[:ond.value])
    out = DeviceArray(shape, a.dtype, a.ctx)
    check(lib.fg_einsum(a.ctx.handle, _NP2FG[a.dtype], _mode(mode), subscripts.encode(), a.ptr, a.ndim, sa, b.ptr,
                        b.ndim, sb, out.ptr, osh, C.byref(ond), None), "einsum")
    a.ctx.sync()
    return out


def matrix_power(a, exponent, mode=PLAIN):
    """A^exponent for a square 2-D DeviceArray (solve.rs:456)."""
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ShapeMismatch(f"matrix_power requires a square matrix, got {'x'.join(map(str, a.shape))}")
    out = DeviceArray(a.shape, a.dtype, a.ctx)
    check(a.ctx._lib.fg_matrix_power(a.ctx.handle, _NP2FG[a.dtype], _mode(mode), a.shape[0], a.ptr,
                                     int(exponent), out.ptr, None), "matrix_power")
    a.ctx.sync()
    return out


def _trsm(np_t, scalar_t, upper, m, n, alpha, a, lda, b, ldb, unit_diag, mode):
    """Shared body of the trsm_left_* mirrors (trsm.rs:46-133): B (m x n,
    row stride ldb) is overwritten by X with op(A) X = alpha B.  Device
    arrays are solved in place; host arrays are staged through the device."""
    if m == 0 or n == 0:
        return
    if lda < m or ldb < n:
        raise ShapeMismatch("trsm: lda must be >= m and ldb >= n")
    _need(a, (m - 1) * lda + m, np_t, "a")
    _need(b, (m - 1) * ldb + n, np_t, "b")
    ctx = default_context()
    lib = ctx._lib
    al = scalar_t(alpha)
    fgdt = L.FG_F64 if np_t == np.float64 else L.FG_F32
    if _is_dev(a) != _is_dev(b):
        raise InvalidValue("mix of device and host operands")
    if _is_dev(a):
        check(lib.fg_trsm_left(ctx.handle, fgdt, _mode(mode), int(upper), int(bool(unit_diag)), m, n,
                               C.byref(al), a.ptr, lda, b.ptr, ldb, None), "trsm")
        ctx.sync()
        return
    da = DeviceArray.from_numpy(a, ctx)
    db = DeviceArray.from_numpy(b, ctx)
    try:
        check(lib.fg_trsm_left(ctx.handle, fgdt, _mode(mode), int(upper), int(bool(unit_diag)), m, n,
                               C.byref(al), da.ptr, lda, db.ptr, ldb, None), "trsm")
        b[...] = db.to_numpy().reshape(b.shape)
    finally:
        da.free()
        db.free()


def trsm_left_lower_f64(m, n, alpha, a, lda, b, ldb, unit_diag, mode=PLAIN):
    """Solve L X = alpha B in place (trsm.rs:46); L lower triangular."""
    _trsm(np.float64, C.c_double, False, m, n, alpha, a, lda, b, ldb, unit_diag, mode)


def trsm_left_upper_f64(m, n, alpha, a, lda, b, ldb, unit_diag, mode=PLAIN):
    """Solve U X = alpha B in place (trsm.rs:70); U upper triangular."""
    _trsm(np.float64, C.c_double, True, m, n, alpha, a, lda, b, ldb, unit_diag, mode)


def trsm_left_lower_f32(m, n, alpha, a, lda, b, ldb, unit_diag, mode=PLAIN):
    """f32 sibling of trsm_left_lower_f64 (trsm.rs:94)."""
    _trsm(np.float32, C.c_float, False, m, n, alpha, a, lda, b, ldb, unit_diag, mode)


def trsm_left_upper_f32(m, n, alpha, a, lda, b, ldb, unit_diag, mode=PLAIN):
    """f32 sibling of trsm_left_upper_f64 (trsm.rs:118)."""
    _trsm(np.float32, C.c_float, True, m, n, alpha, a, lda, b, ldb, unit_diag, mode)


TUNE_OPS = {"i8": 0, "split_f32": 1, "f64": 2, "f32": 3}


def tune_lookup(op, m, n, k):
    """(variant, splits) the autotuned table picks for a problem size."""
    v, s = C.c_int(), C.c_int()
    check(L.load().fg_tune_lookup(TUNE_OPS[op], m, n, k, C.byref(v), C.byref(s)), "tune_lookup")
    return v.value, s.value


class tune_forced:
    """Context manager forcing (variant, splits) for one family, process-wide
    (the autotuner's and the tests' way to reach every variant)."""

    def __init__(self, op, variant, splits=1):
        self.op, self.variant, self.splits = TUNE_OPS[op], variant, splits

    def __enter__(self):
        check(L.load().fg_tune_force(self.op, self.variant, self.splits), "tune_force")
        return self

    def __exit__(self, *exc):
        L.load().fg_tune_force(self.op, -1, 1)
        return False


def _shard(dims, weights, world, rank, policy):
    if world < 1 or not 0 <= rank < world:
        raise InvalidValue(f"rank {rank} outside a world of {world}")
    d = np.ascontiguousarray(np.asarray(dims, dtype=np.int64).reshape(-1, 3))
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    out = np.empty(len(d), np.int64)
    cnt = C.c_size_t()
    check(L.load().fg_shard_plan(d.ctypes.data, None if w is None else w.ctypes.data, len(d), world, rank,
                                 policy, out.ctypes.data, C.byref(cnt)), "shard_plan")
    return [int(x) for x in out[:cnt.value]]


def shard_problems(dims, world, rank):
    """Indices of the problems of a ragged batch (rows of (m, n, k)) that rank
    `rank` of `world` runs (fg_shard_plan, FG_SHARD_LPT): heaviest first by
    2mnk, each problem to the least-loaded rank so far (lowest rank on
    ties).  Every rank computes the same assignment from the same table, so
    sharding a batch across GPUs needs no communication; the shards are
    disjoint, cover every problem, and differ in load by at most one
    problem's work."""
    return _shard(dims, None, world, rank, L.FG_SHARD_LPT)


def shard_requests(dims, world, rank, weights=None):
    """Indices of the requests of a served stream (rows of (m, n, k) in
    arrival order) that rank `rank` of `world` serves (FG_SHARD_ONLINE): each
    request to the rank with the least cost so far -- `weights` (estimated
    seconds, say) or 2mnk -- so a rank can route a request as it arrives."""
    return _shard(dims, weights, world, rank, L.FG_SHARD_ONLINE)


def _grouped_dtype(dtype):
    d = np.dtype(dtype)
    return L.FG_I8 if d == np.int8 else L.FG_U8I8 if d == np.uint8 else L.FG_F32


def gemm_grouped(problems, dtype=np.float32, mode=PLAIN):
    """One persistent grouped launch over ragged problems
    [(m, n, k, A, B, C), ...] or [(m, n, k, A, B, C, lda, ldb, ldc), ...]
    (DeviceArrays or raw device pointers; leading dimensions in elements,
    default k, n, n).  dtype int8: i8 x i8; uint8: u8 x i8; float32."""
    ctx = default_context()
    dt = _grouped_dtype(dtype)
    tab = _table(problems)
    check(ctx._lib.fg_gemm_grouped(ctx.handle, dt, _mode(mode), tab, len(problems), None),
          "grouped")
    ctx.sync()


class GroupedPlan:
    """Prepared grouped batch replayed from a CUDA graph."""

    def __init__(self, problems, dtype=np.float32, mode=PLAIN):
        self.ctx = default_context()
        dt = _grouped_dtype(dtype)
        self._tab = _table(problems)
        h = C.c_void_p()
        check(self.ctx._lib.fg_grouped_plan_create(self.ctx.handle, dt, _mode(mode), self._tab,
                                                   len(problems), None, C.byref(h)), "plan")
        self.handle = h

    def run(self, sync=True):
        check(self.ctx._lib.fg_grouped_plan_run(self.handle, None), "plan run")
        if sync:
            self.ctx.sync()

    def close(self):
        if self.handle:
            self.ctx._lib.fg_grouped_plan_destroy(self.handle)
            self.handle = None


_REQ_DTYPE = {np.dtype(np.float64): L.FG_F64, np.dtype(np.float32): L.FG_F32,
              np.dtype(np.complex128): L.FG_C64, np.dtype(np.complex64): L.FG_C32,
              np.dtype(np.int8): L.FG_I8, np.dtype(np.uint8): L.FG_U8I8,
              np.dtype(np.int16): L.FG_I16}


class Server:
    """Continuous-batching matmul server (fg_server_*): requests are
    C = A @ B on DeviceArrays; many host threads may submit concurrently."""

    def __init__(self, hbm_budget_bytes=40 << 30, streams=4, max_group=256, ctx=None):
        self.ctx = ctx or default_context()
        self._lib = self.ctx._lib
        h = C.c_void_p()
        check(self._lib.fg_server_start(self.ctx.handle, int(hbm_budget_bytes), int(streams),
                                        int(max_group), C.byref(h)), "fg_server_start")
        self.handle = h

    def submit(self, a, b, c, mode=PLAIN):
        m, k = a.shape
        n = b.shape[1]
        dt = _REQ_DTYPE[np.dtype(a.dtype)]
        req = L.fg_request(dt, _mode(mode), m, n, k, a.ptr, b.ptr, c.ptr, 0)
        t = C.c_uint64()
        check(self._lib.fg_server_submit(self.handle, C.byref(req), C.byref(t)), "submit")
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        check(self._lib.fg_server_wait(self.handle, ticket, int(timeout_ms)), "wait")

    def wait_times(self, ticket, timeout_ms=-1):
        """wait(), returning (submitted, completed) in seconds of clock()."""
        t0, t1 = C.c_double(), C.c_double()
        check(self._lib.fg_server_wait_times(self.handle, ticket, int(timeout_ms), C.byref(t0), C.byref(t1)),
              "wait")
        return t0.value, t1.value

    def clock(self):
        """The server's monotonic clock (seconds)."""
        return self._lib.fg_server_clock()

    def stats(self):
        s = L.fg_server_stats()
        check(self._lib.fg_server_stats_get(self.handle, C.byref(s)), "stats")
        return {f: getattr(s, f) for f, _ in L.fg_server_stats._fields_}

    def stop(self):
        if getattr(self, "handle", None):
            self._lib.fg_server_stop(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
