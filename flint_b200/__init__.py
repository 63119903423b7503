"""flint_b200 -- B200 small-prime NTT multiplication (FLINT fft_small, mpn_ctx route).

Python mirror of the C ABI in include/gpu_fft_small.h, bound with ctypes to
the in-tree CUDA library libflint_b200.so.  Names follow the reference's
functions (src/fft_small.h):

    MpnCtx(p)                      mpn_ctx_init / mpn_ctx_clear
    MpnCtx.mpn_mul(a, b)           mpn_ctx_mpn_mul
    MpnCtx.mpn_mul_range(..)       _mpn_ctx_mpn_mul_range
    MpnCtx.nmod_poly_mul_mid(..)   _nmod_poly_mul_mid_mpn_ctx
    MpnCtx.fmpz_poly_mul_mid(..)   _fmpz_poly_mul_mid_mpn_ctx (raw coefficient rows)
    MpnBatch(ctx, reqs)            batches of uneven products (no counterpart)
    MpnPipe(depth)                 streams of host-pointer products (no counterpart)
    MpnCtx.mpn_mul_device(..)      device-pointer twin (no host copies)
    mpn_mul_plan, mpn_mul_split_plan   plan introspection

There is no CPU fallback: if the library or a GPU is missing, every call
raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# FLINT_B200_LIB selects another build of the library (same C ABI), e.g. one
# compiled with different options; the default is the in-tree build.
LIB_PATH = os.environ.get("FLINT_B200_LIB") or os.path.join(_HERE, "libflint_b200.so")
DEFAULT_PRIME = 0x0003F00000000001

OK, EINVAL, ETOOBIG, ECUDA, ETIMEOUT, ENOPRIMES = 0, 1, 2, 3, 4, 5

_lib = None


class GpuFftSmallError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("gpu_fft_small error %d: %s" % (code, msg))
        self.code = code


class _Ctx(ctypes.Structure):
    _fields_ = [("impl", ctypes.c_void_p)]


class _Pipe(ctypes.Structure):
    """gpu_mpn_pipe_struct"""
    _fields_ = [("impl", ctypes.c_void_p)]


class _Nmod(ctypes.Structure):
    _fields_ = [("n", ctypes.c_ulong), ("ninv", ctypes.c_ulong), ("norm", ctypes.c_ulong)]


class _MulPrecomp(ctypes.Structure):
    _fields_ = [("impl", ctypes.c_void_p), ("bn", ctypes.c_ulong), ("btrunc", ctypes.c_ulong),
                ("depth", ctypes.c_ulong)]


class _DivremPrecomp(ctypes.Structure):
    _fields_ = [("quo_maker", _MulPrecomp), ("rem_maker", _MulPrecomp)]


class MulReq(ctypes.Structure):
    """gpu_mpn_mul_req: one product z = a * b of a batch (device pointers)."""
    _fields_ = [("z", ctypes.c_void_p), ("a", ctypes.c_void_p), ("an", ctypes.c_ulong),
                ("b", ctypes.c_void_p), ("bn", ctypes.c_ulong)]


class FmpzMulReq(ctypes.Structure):
    """gpu_fmpz_mul_req: one integer-polynomial window product of a list
    (device pointers; raw two's complement coefficient rows)."""
    _fields_ = [("z", ctypes.c_void_p), ("zw", ctypes.c_ulong), ("zl", ctypes.c_ulong),
                ("zh", ctypes.c_ulong), ("a", ctypes.c_void_p), ("aw", ctypes.c_ulong),
                ("an", ctypes.c_ulong), ("b", ctypes.c_void_p), ("bw", ctypes.c_ulong),
                ("bn", ctypes.c_ulong)]


class MulConfig(ctypes.Structure):
    """gpu_mul_config: route, prime count, log2 transform length, log2 row
    length, flags (FLAG_THREE: a 3 2^(logM-2)-point transform; FLAG_SPLIT:
    chunks of the long operand against the short one)."""
    _fields_ = [("route", ctypes.c_int), ("np", ctypes.c_int), ("logM", ctypes.c_int),
                ("logC", ctypes.c_int), ("flags", ctypes.c_int)]

    def key(self):
        return (self.route, self.np, self.logM, self.logC, self.flags)

    def __repr__(self):
        return "MulConfig(route=%d, np=%d, logM=%d, logC=%d, flags=%d)" % self.key()


ROUTE_NTT, ROUTE_BASECASE = 0, 1
FLAG_THREE, FLAG_SPLIT, FLAG_ROWS16, FLAG_ROWS32 = 1, 2, 4, 8


class BatchOptions(ctypes.Structure):
    """gpu_mpn_batch_options: schedule knobs of a batch."""
    _fields_ = [("promote_small", ctypes.c_int), ("max_streams", ctypes.c_int),
                ("use_graph", ctypes.c_int)]


# symbol -> (restype, argtypes); every symbol include/gpu_fft_small.h declares
_P = ctypes.c_void_p
_U = ctypes.c_ulong
_S = ctypes.c_long
_CTX = ctypes.POINTER(_Ctx)
_PIPE = ctypes.POINTER(_Pipe)
SIGNATURES = {
    "gpu_mpn_ctx_init": (None, [_CTX, _U]),
    "gpu_mpn_ctx_init_status": (ctypes.c_int, [_CTX, _U]),
    "gpu_mpn_ctx_clear": (None, [_CTX]),
    "gpu_mpn_ctx_mpn_mul": (None, [_CTX, _P, _P, _U, _P, _U]),
    "gpu_mpn_ctx_mpn_mul_status": (ctypes.c_int, [_CTX, _P, _P, _U, _P, _U]),
    "gpu_mpn_pipe_init": (ctypes.c_int, [_PIPE, ctypes.c_int]),
    "gpu_mpn_pipe_submit": (ctypes.c_int, [_PIPE, _P, _P, _U, _P, _U, ctypes.POINTER(ctypes.c_longlong)]),
    "gpu_mpn_pipe_wait": (ctypes.c_int, [_PIPE, ctypes.c_longlong]),
    "gpu_mpn_pipe_clear": (None, [_PIPE]),
    "gpu_test_crt_lookback_timeout": (ctypes.c_int, [_CTX]),
    "gpu_test_set_device_error": (ctypes.c_int, [_CTX]),
    "gpu_test_pipe_slot_ctx": (ctypes.c_void_p, [_PIPE, ctypes.c_int]),
    "_gpu_mpn_ctx_mpn_mul_range": (None, [_CTX, _P, _U, _U, _P, _U, _P, _U]),
    "gpu_mpn_mul_device": (ctypes.c_int, [_CTX, _P, _P, _U, _P, _U, _P]),
    "gpu_mpn_mul_device_noalloc": (ctypes.c_int, [_P, _P, _U, _P, _U, _P]),
    "gpu_mpn_mul_range_device": (ctypes.c_int, [_CTX, _P, _U, _U, _P, _U, _P, _U, _P]),
    "gpu_mpn_mulmid_default_mpn_ctx": (None, [_P, _P, _S, _P, _S, _S, _S]),
    "_gpu_nmod_poly_mul_mid_mpn_ctx": (None, [_P, _U, _U, _P, _U, _P, _U, _Nmod, _CTX]),
    "_gpu_nmod_poly_mul_mid_status": (ctypes.c_int, [_P, _U, _U, _P, _U, _P, _U, _Nmod, _CTX]),
    "gpu_nmod_poly_mul_mid_device": (ctypes.c_int, [_CTX, _P, _U, _U, _P, _U, _P, _U, _Nmod, _P]),
    "_gpu_nmod_poly_divrem_mpn_ctx": (None, [_P, _P, _P, _U, _P, _U, _Nmod, _CTX]),
    "_gpu_nmod_poly_divrem_status": (ctypes.c_int, [_P, _P, _P, _U, _P, _U, _Nmod, _CTX]),
    "gpu_get_default_mpn_ctx": (_CTX, []),
    "gpu_butterfly_rate": (ctypes.c_int, [_CTX, ctypes.POINTER(ctypes.c_double)]),
    "gpu_mul_precomp_init_status": (ctypes.c_int, [_P, _P, _U, _U, _U, _Nmod, _CTX]),
    "_gpu_mul_precomp_init": (None, [_P, _P, _U, _U, _U, _Nmod, _CTX]),
    "_gpu_mul_precomp_clear": (None, [_P]),
    "_gpu_nmod_poly_mul_mid_precomp": (ctypes.c_int, [_P, _U, _U, _P, _U, _P, _Nmod, _CTX]),
    "gpu_nmod_poly_mul_mid_precomp_device": (ctypes.c_int, [_P, _U, _U, _P, _U, _P, _P]),
    "_gpu_nmod_poly_divrem_precomp_init_status": (ctypes.c_int, [_P, _P, _U, _U, _Nmod, _CTX]),
    "_gpu_nmod_poly_divrem_precomp_init": (None, [_P, _P, _U, _U, _Nmod, _CTX]),
    "_gpu_nmod_poly_divrem_precomp": (ctypes.c_int, [_P, _P, _P, _U, _P, _Nmod, _CTX]),
    "gpu_nmod_poly_divrem_precomp_device": (ctypes.c_int, [_P, _P, _P, _U, _P, _P]),
    "_gpu_nmod_poly_divrem_precomp_clear": (None, [_P]),
    "gpu_mulmod_2expp1_ctx_init_status": (ctypes.c_int, [_P, _CTX, _S, _S]),
    "gpu_mulmod_2expp1_ctx_init": (None, [_P, _CTX, _S, _S]),
    "gpu_mulmod_2expp1_ctx_clear": (None, [_P]),
    "gpu_mulmod_2expp1_ctx_info": (ctypes.c_int, [_P, _P, _P, _P, _P]),
    "gpu_mulmod_2expp1_choose_np": (_S, [_S, _S]),
    "gpu_mulmod_2expp1_status": (ctypes.c_int, [_P, _P, _P, _P]),
    "gpu_mulmod_2expp1": (None, [_P, _P, _P, _P]),
    "gpu_mulmod_2expp1_batch_device": (ctypes.c_int, [_P, _P, _P, _P, _U, _U, _P]),
    "gpu_mulmod_2expp1_transformed_size": (_S, [_P, _U]),
    "gpu_mulmod_2expp1_transform_device": (ctypes.c_int, [_P, _P, _P, _U, _U, _P]),
    "gpu_mulmod_2expp1_mul_cached_device": (ctypes.c_int, [_P, _P, _P, _P, _U, _U, _P]),
    "gpu_mulmod_2expp1_transform": (ctypes.c_int, [_P, _P, _P]),
    "gpu_mulmod_2expp1_mul_cached": (ctypes.c_int, [_P, _P, _P, _P]),
    "gpu_default_mpn_ctx_cleanup": (None, []),
    "gpu_mpn_mul_default_mpn_ctx": (None, [_P, _P, _S, _P, _S]),
    "_gpu_nmod_poly_mul_mid_default_mpn_ctx": (None, [_P, _S, _S, _P, _S, _P, _S, _Nmod]),
    "_gpu_fmpz_poly_mul_mid_mpn_ctx": (ctypes.c_int, [_P, _U, _U, _P, _U, _P, _U, _CTX]),
    "_gpu_fmpz_poly_mul_mid_default_mpn_ctx": (ctypes.c_int, [_P, _S, _S, _P, _S, _P, _S]),
    "gpu_fmpz_set_signed_hook": (None, [_P]),
    "_gpu_fmpz_poly_mul_mid_raw": (ctypes.c_int, [_P, _U, _U, _U, _P, _U, _U, _P, _U, _U, _CTX]),
    "gpu_fmpz_poly_mul_mid_device": (ctypes.c_int, [_CTX, _P, _U, _U, _U, _P, _U, _U, _P, _U,
                                                    _U, _P]),
    "gpu_mpn_mul_config_resolve": (ctypes.c_int, [_U, _U, ctypes.POINTER(MulConfig)]),
    "gpu_mpn_mul_device_config": (ctypes.c_int, [_CTX, _P, _P, _U, _P, _U,
                                                 ctypes.POINTER(MulConfig), _P]),
    "gpu_fmpz_poly_mul_config_resolve": (ctypes.c_int, [_U, _U, _U, _U, ctypes.POINTER(MulConfig)]),
    "gpu_fmpz_poly_mul_mid_device_config": (ctypes.c_int, [_CTX, _P, _U, _U, _U, _P, _U, _U, _P, _U,
                                                           _U, ctypes.POINTER(MulConfig), _P]),
    "gpu_fmpz_poly_mul_mid_device_list": (ctypes.c_int, [_CTX, _P, ctypes.c_size_t, _P, _P]),
    "gpu_mpn_mul_device_list": (ctypes.c_int, [_CTX, _P, ctypes.c_size_t, _P, _P]),
    "gpu_mul_reference_rule": (ctypes.c_int, [ctypes.c_int, _U, _U, _U, _U, ctypes.POINTER(MulConfig)]),
    "gpu_mul_time_config": (ctypes.c_int, [_CTX, ctypes.c_int, _U, _U, _U, _U,
                                           ctypes.POINTER(MulConfig), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double)]),
    "gpu_mpn_mul_time_batched": (ctypes.c_int, [_CTX, _U, _U, ctypes.POINTER(MulConfig), ctypes.c_int,
                                                ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "gpu_mlp_init": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.c_ulonglong]),
    "gpu_mlp_nparams": (ctypes.c_int, [_P]),
    "gpu_mlp_get_params": (ctypes.c_int, [_P, _P, ctypes.c_size_t]),
    "gpu_mlp_set_params": (ctypes.c_int, [_P, _P, ctypes.c_size_t]),
    "gpu_mlp_predict": (ctypes.c_int, [_P, _P, ctypes.c_int, _P]),
    "gpu_mlp_predict_device": (ctypes.c_int, [_P, _P, ctypes.c_int, _P, _P]),
    "gpu_mlp_gradient": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, _P, _P]),
    "gpu_mlp_train": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_ulonglong, _P]),
    "gpu_mlp_clear": (None, [_P]),
    "gpu_fft_plan_init_mpn": (ctypes.c_int, [ctypes.POINTER(_P), _CTX, _U, _U, _U, ctypes.c_int]),
    "gpu_fft_plan_init_nmod": (ctypes.c_int, [ctypes.POINTER(_P), _CTX, _U, _U, _U, _U, _U, _Nmod]),
    "gpu_fft_plan_init_mpn_np": (ctypes.c_int, [ctypes.POINTER(_P), _CTX, _U, _U, _U, ctypes.c_int, ctypes.c_int]),
    "gpu_fft_plan_init_nmod_cyclic": (ctypes.c_int, [ctypes.POINTER(_P), _CTX, _U, _U, _U, _U, _Nmod]),
    "gpu_fft_plan_init_mpn_cyclic": (ctypes.c_int, [ctypes.POINTER(_P), _CTX, ctypes.POINTER(_U), _U]),
    "gpu_fft_op_sizeof_data": (_U, [_P]),
    "gpu_fft_op_init_borrowed": (ctypes.c_int, [ctypes.POINTER(_P), _P, _P]),
    "gpu_fft_export_mpn_signed": (ctypes.c_int, [_P, _U, ctypes.POINTER(ctypes.c_int), _P, _U, _P, _P]),
    "gpu_fft_export_mpn_signed_trunc": (ctypes.c_int, [_P, _U, ctypes.POINTER(ctypes.c_int), _P, _U, _U, _P,
                                                        _P]),
    "gpu_fft_plan_info": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "gpu_fft_plan_clear": (None, [_P]),
    "gpu_fft_op_init": (ctypes.c_int, [ctypes.POINTER(_P), _P]),
    "gpu_fft_op_clear": (None, [_P]),
    "gpu_fft_fft_mpn": (ctypes.c_int, [_P, _P, _U, _P, _P]),
    "gpu_fft_fft_nmod": (ctypes.c_int, [_P, _P, _U, _P, _P]),
    "gpu_fft_op_pointwise": (ctypes.c_int, [ctypes.c_int, _P, _P, _P, _P, _P]),
    "gpu_fft_ifft": (ctypes.c_int, [_P, _P, _P]),
    "gpu_fft_export_mpn": (ctypes.c_int, [_P, _U, _P, _P, _P]),
    "gpu_fft_export_nmod": (ctypes.c_int, [_P, _U, _U, _P, _Nmod, _P, _P]),
    "gpu_fft_op_check": (ctypes.c_int, [_P, _P]),
    "gpu_mpn_batch_init": (ctypes.c_int, [ctypes.POINTER(_P), _CTX, _P, ctypes.c_size_t, _P]),
    "gpu_mpn_batch_init_config": (ctypes.c_int, [ctypes.POINTER(_P), _CTX, _P, _P, ctypes.c_size_t,
                                                 _P]),
    "gpu_mpn_batch_run": (ctypes.c_int, [_P, _P]),
    "gpu_mpn_batch_check": (ctypes.c_int, [_P, _P]),
    "gpu_mpn_batch_launches": (ctypes.c_int, [_P]),
    "gpu_mpn_batch_classes": (ctypes.c_int, [_P]),
    "gpu_mpn_batch_clear": (None, [_P]),
    "gpu_fft_small_set_throw": (None, [_P]),
    "gpu_fft_small_last_error": (ctypes.c_char_p, []),
    "gpu_mpn_mul_plan": (ctypes.c_int, [_U, _U, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]),
    "gpu_mpn_mul_split_plan": (ctypes.c_int, [_U, _U, ctypes.POINTER(ctypes.c_int)]),
    "gpu_mpn_mul_transform_points": (ctypes.c_int, [_U, _U, ctypes.c_int, ctypes.POINTER(_U)]),
    "gpu_fft_small_prime": (_U, [ctypes.c_int]),
    "gpu_mpn_ctx_last_launches": (ctypes.c_int, [_CTX]),
    "gpu_mpn_ctx_set_timing": (ctypes.c_int, [_CTX, ctypes.c_int]),
    "gpu_mpn_ctx_kernel_times": (ctypes.c_int, [_CTX, ctypes.POINTER(ctypes.c_double),
                                                ctypes.POINTER(ctypes.c_long), ctypes.c_int]),
}

KERNEL_SLOTS = ("k_fwd_cols", "k_rows", "k_inv_cols", "k_crt_carry")


def lib():
    """Load libflint_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libflint_b200.so is not built; run "
                              "`python -m flint_b200.build` (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != OK:
        raise GpuFftSmallError(rc, lib().gpu_fft_small_last_error().decode())


def _limbs(x):
    x = np.ascontiguousarray(x, dtype=np.uint64)
    if x.ndim != 1:
        raise ValueError("limb arrays are one-dimensional")
    return x


def mpn_mul_plan(an, bn):
    """(number of primes, log2 transform length) the GPU path uses."""
    np_, lm = ctypes.c_int(), ctypes.c_int()
    _check(lib().gpu_mpn_mul_plan(an, bn, ctypes.byref(np_), ctypes.byref(lm)))
    return np_.value, lm.value


def mpn_mul_split_plan(an, bn):
    """log2 chunk transform length of a split an x bn product, 0 if not split."""
    lc = ctypes.c_int()
    _check(lib().gpu_mpn_mul_split_plan(an, bn, ctypes.byref(lc)))
    return lc.value


def mpn_mul_transform_points(an, bn, square=False):
    """Points of the cyclic transform a whole an x bn product runs under the
    default plan (2^logM, 3 2^(logM-2), a split chunk's length, or 0 for the
    basecase route)."""
    v = _U()
    _check(lib().gpu_mpn_mul_transform_points(an, bn, 1 if square else 0, ctypes.byref(v)))
    return v.value


def prime(i):
    return int(lib().gpu_fft_small_prime(i))


def resolve_config(kind, an, bn, cfg=None, aw=1, bw=1):
    """The full configuration (defaults filled in) for a product, or raises
    GpuFftSmallError if cfg is invalid for it."""
    c = MulConfig(*(cfg.key() if cfg is not None else (0, 0, 0, 0, 0)))
    if kind == 0:
        _check(lib().gpu_mpn_mul_config_resolve(an, bn, ctypes.byref(c)))
    else:
        _check(lib().gpu_fmpz_poly_mul_config_resolve(an, aw, bn, bw, ctypes.byref(c)))
    return c


def reference_rule(kind, an, bn, aw=1, bw=1):
    """The configuration the reference's profile choice (mpn_ctx_best_profile)
    makes in this configuration space (gpu_mul_reference_rule)."""
    c = MulConfig()
    _check(lib().gpu_mul_reference_rule(kind, an, aw, bn, bw, ctypes.byref(c)))
    return c


class Mlp:
    """The cost model's network (gpu_mlp_*): n_in -> 3 x 64 ReLU -> 1, fp32,
    trained and evaluated by the library's CUDA kernels."""

    def __init__(self, n_in, seed=1):
        self.n_in = n_in
        self._h = ctypes.c_void_p()
        _check(lib().gpu_mlp_init(ctypes.byref(self._h), n_in, seed))
        self.nparams = int(lib().gpu_mlp_nparams(self._h))

    def params(self):
        p = np.empty(self.nparams, dtype=np.float32)
        _check(lib().gpu_mlp_get_params(self._h, p.ctypes.data, self.nparams))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib().gpu_mlp_set_params(self._h, p.ctypes.data, len(p)))

    def predict(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.empty(len(X), dtype=np.float32)
        _check(lib().gpu_mlp_predict(self._h, X.ctypes.data, len(X), y.ctypes.data))
        return y

    def gradient(self, X, t):
        X = np.ascontiguousarray(X, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.nparams, dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().gpu_mlp_gradient(self._h, X.ctypes.data, t.ctypes.data, len(X), g.ctypes.data,
                                      ctypes.byref(loss)))
        return g, loss.value

    def train(self, X, t, epochs=200, batch=256, lr=1e-3, seed=7):
        X = np.ascontiguousarray(X, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().gpu_mlp_train(self._h, X.ctypes.data, t.ctypes.data, len(X), epochs, batch, lr,
                                   seed, ctypes.byref(loss)))
        return loss.value

    def close(self):
        if self._h:
            lib().gpu_mlp_clear(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _raw_bits(x):
    """Largest magnitude bit count over the rows of a two's complement array."""
    if x.size == 0:
        return 0
    w = x.shape[1]
    neg = (x[:, -1] >> np.uint64(63)).astype(bool)
    best = 0
    for row, s in zip(x, neg):
        v = int.from_bytes(row.tobytes(), "little")
        if s:
            v = (1 << (64 * w)) - v
        best = max(best, v.bit_length())
    return best


def fmpz_result_width(a, b):
    """Limbs per coefficient that hold every coefficient of a * b."""
    mn = min(len(a), len(b))
    bits = _raw_bits(a) + _raw_bits(b) + (mn - 1).bit_length() + 1
    return max(1, (bits + 63) // 64)


class MpnCtx:
    """GPU counterpart of mpn_ctx_t (src/fft_small.h:382-433)."""

    def __init__(self, p=DEFAULT_PRIME):
        self._c = _Ctx()
        _check(lib().gpu_mpn_ctx_init_status(ctypes.byref(self._c), p))

    @property
    def ptr(self):
        return ctypes.byref(self._c)

    def close(self):
        if self._c.impl:
            lib().gpu_mpn_ctx_clear(ctypes.byref(self._c))
            self._c.impl = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mpn_mul(self, a, b, out=None):
        """a * b as an+bn limbs (mpn_ctx_mpn_mul)."""
        a = _limbs(a)
        b = a if b is a else _limbs(b)
        an, bn = len(a), len(b)
        z = np.empty(an + bn, dtype=np.uint64) if out is None else out
        _check(lib().gpu_mpn_ctx_mpn_mul_status(self.ptr, z.ctypes.data, a.ctypes.data, an,
                                                b.ctypes.data, bn))
        return z

    def mpn_mul_range(self, lo, hi, a, b):
        """limbs [lo, hi) of a * b (_mpn_ctx_mpn_mul_range): exact for lo = 0,
        for lo > 0 a lower approximation short by at most 2 units."""
        a = _limbs(a)
        b = a if b is a else _limbs(b)
        z = np.empty(max(hi - lo, 0), dtype=np.uint64)
        if hi > lo:
            lib()._gpu_mpn_ctx_mpn_mul_range(self.ptr, z.ctypes.data, lo, hi, a.ctypes.data,
                                             len(a), b.ctypes.data, len(b))
        return z

    def mpn_mul_range_device(self, z_ptr, lo, hi, a_ptr, an, b_ptr, bn, stream=None):
        """Queue limbs [lo, hi) of a * b on device pointers (see mpn_mul_range)."""
        _check(lib().gpu_mpn_mul_range_device(self.ptr, z_ptr, lo, hi, a_ptr, an, b_ptr, bn, stream))

    def mpn_mul_device(self, z_ptr, a_ptr, an, b_ptr, bn, stream=None):
        """Queue z = a * b on device pointers (ints); returns without syncing."""
        _check(lib().gpu_mpn_mul_device(self.ptr, z_ptr, a_ptr, an, b_ptr, bn, stream))

    def nmod_poly_mul_mid(self, zl, zh, a, b, n):
        """coefficients [zl, zh) of a * b mod n (_nmod_poly_mul_mid_mpn_ctx)."""
        a = _limbs(a)
        b = a if b is a else _limbs(b)
        z = np.empty(max(zh - zl, 0), dtype=np.uint64)
        _check(lib()._gpu_nmod_poly_mul_mid_status(z.ctypes.data, zl, zh, a.ctypes.data, len(a),
                                                   b.ctypes.data, len(b), _Nmod(n, 0, 0),
                                                   self.ptr))
        return z

    def fmpz_poly_mul_mid(self, zl, zh, a, b, zw=None):
        """coefficients [zl, zh) of a * b for integer polynomials given as
        (n, w) uint64 arrays of two's complement coefficients (raw form of
        _fmpz_poly_mul_mid_mpn_ctx); returns a (zh - zl, zw) array."""
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = a if b is a else np.ascontiguousarray(b, dtype=np.uint64)
        (an, aw), (bn, bw) = a.shape, b.shape
        if zw is None:
            zw = fmpz_result_width(a, b)
        z = np.empty((max(zh - zl, 0), zw), dtype=np.uint64)
        _check(lib()._gpu_fmpz_poly_mul_mid_raw(z.ctypes.data, zw, zl, zh, a.ctypes.data, aw, an,
                                                b.ctypes.data, bw, bn, self.ptr))
        return z

    def fmpz_poly_mul_device(self, z_ptr, zw, zl, zh, a_ptr, aw, an, b_ptr, bw, bn, stream=None):
        """Queue the raw-form window product on device pointers."""
        _check(lib().gpu_fmpz_poly_mul_mid_device(self.ptr, z_ptr, zw, zl, zh, a_ptr, aw, an,
                                                  b_ptr, bw, bn, stream))

    def nmod_poly_mul_mid_device(self, z_ptr, zl, zh, a_ptr, an, b_ptr, bn, n, stream=None):
        """Queue coefficients [zl, zh) of a * b mod n on device pointers (ints)."""
        _check(lib().gpu_nmod_poly_mul_mid_device(self.ptr, z_ptr, zl, zh, a_ptr, an, b_ptr, bn,
                                                  _Nmod(n, 0, 0), stream))

    def mpn_mul_device_config(self, z_ptr, a_ptr, an, b_ptr, bn, cfg, stream=None):
        """mpn_mul_device under an explicit MulConfig."""
        _check(lib().gpu_mpn_mul_device_config(self.ptr, z_ptr, a_ptr, an, b_ptr, bn,
                                               ctypes.byref(cfg), stream))

    def fmpz_poly_mul_device_config(self, z_ptr, zw, zl, zh, a_ptr, aw, an, b_ptr, bw, bn, cfg,
                                    stream=None):
        _check(lib().gpu_fmpz_poly_mul_mid_device_config(self.ptr, z_ptr, zw, zl, zh, a_ptr, aw,
                                                         an, b_ptr, bw, bn, ctypes.byref(cfg),
                                                         stream))

    def mpn_mul_device_list(self, reqs, cfgs=None, stream=None):
        """Queue a list of whole products (MulReq or (z, a, an, b, bn) tuples of
        device pointers) with one call, each as mpn_mul_device would run it."""
        n = len(reqs)
        arr = (MulReq * n)(*[r if isinstance(r, MulReq) else MulReq(*r) for r in reqs])
        carr = (MulConfig * n)(*cfgs) if cfgs is not None else None
        _check(lib().gpu_mpn_mul_device_list(self.ptr, arr, n, carr, stream))

    def fmpz_poly_mul_device_list(self, reqs, cfgs=None, stream=None):
        """Queue a list of integer-polynomial window products (FmpzMulReq,
        device pointers) with one call; cfgs: None or one MulConfig per
        request."""
        n = len(reqs)
        arr = (FmpzMulReq * n)(*reqs)
        carr = (MulConfig * n)(*cfgs) if cfgs is not None else None
        _check(lib().gpu_fmpz_poly_mul_mid_device_list(self.ptr, arr, n, carr, stream))

    def time_config(self, kind, an, bn, cfg=None, aw=1, bw=1, reps=3):
        """Median device milliseconds of a product under cfg (autotuner probe)."""
        ms = ctypes.c_double()
        _check(lib().gpu_mul_time_config(self.ptr, kind, an, aw, bn, bw,
                                         ctypes.byref(cfg) if cfg is not None else None, reps,
                                         ctypes.byref(ms)))
        return ms.value

    def time_batched(self, an, bn, cfg=None, copies=16, reps=3):
        """Marginal device milliseconds of an an x bn product inside a batch of
        `copies` such products under cfg (autotuner probe)."""
        ms = ctypes.c_double()
        _check(lib().gpu_mpn_mul_time_batched(self.ptr, an, bn,
                                              ctypes.byref(cfg) if cfg is not None else None,
                                              copies, reps, ctypes.byref(ms)))
        return ms.value

    def nmod_poly_divrem(self, a, b, n):
        """(q, r) with a = q b + r mod n, deg r < deg b (_nmod_poly_divrem_mpn_ctx)."""
        a, b = _limbs(a), _limbs(b)
        q = np.empty(len(a) - len(b) + 1, dtype=np.uint64)
        r = np.empty(len(b) - 1, dtype=np.uint64)
        _check(lib()._gpu_nmod_poly_divrem_status(q.ctypes.data, r.ctypes.data, a.ctypes.data, len(a),
                                                  b.ctypes.data, len(b), _Nmod(n, 0, 0), self.ptr))
        return q, r

    @property
    def last_launches(self):
        return int(lib().gpu_mpn_ctx_last_launches(self.ptr))

    def butterfly_rate(self):
        """Measured 31-bit butterflies per second from registers (gpu_butterfly_rate)."""
        v = ctypes.c_double()
        _check(lib().gpu_butterfly_rate(self.ptr, ctypes.byref(v)))
        return v.value

    def set_timing(self, on=True):
        """Per-kernel CUDA-event timing on the launching stream (resets totals)."""
        _check(lib().gpu_mpn_ctx_set_timing(self.ptr, 1 if on else 0))

    def kernel_times(self):
        """{kernel: (total ms, launches)} since the last set_timing()."""
        ms = (ctypes.c_double * 8)()
        cnt = (ctypes.c_long * 8)()
        n = lib().gpu_mpn_ctx_kernel_times(self.ptr, ms, cnt, 8)
        return {KERNEL_SLOTS[k]: (ms[k], cnt[k]) for k in range(n)}


class MpnPipe:
    """A pipeline of host-pointer products (gpu_mpn_pipe_*): `depth` slots
    take submitted products in turn, so one product's download, the next
    one's upload and another one's kernels overlap.  submit() returns a
    ticket at once; wait(ticket) returns the product (the array z) when it
    is complete.  The operand and output arrays are kept referenced until
    their ticket is waited for; pinned host memory (e.g. torch's
    pin_memory()) makes the copies asynchronous."""

    def __init__(self, depth=2):
        self._c = _Pipe()
        _check(lib().gpu_mpn_pipe_init(ctypes.byref(self._c), depth))
        self.depth = depth
        self._held = {}

    def submit(self, a, b, out=None):
        """Queue a * b; a, b, out: 1-D uint64 arrays or pinned torch int64
        tensors (then out is required).  Returns the ticket."""
        if hasattr(a, "data_ptr"):
            an, bn = a.numel(), b.numel()
            pa, pb, pz, z = a.data_ptr(), b.data_ptr(), out.data_ptr(), out
            if out.numel() < an + bn:
                raise ValueError("output shorter than an + bn")
        else:
            a = _limbs(a)
            b = a if b is a else _limbs(b)
            an, bn = len(a), len(b)
            z = np.empty(an + bn, dtype=np.uint64) if out is None else out
            if len(z) < an + bn or z.dtype != np.uint64 or not z.flags.c_contiguous:
                raise ValueError("output must be a contiguous uint64 array of an + bn limbs")
            pa, pb, pz = a.ctypes.data, b.ctypes.data, z.ctypes.data
        t = ctypes.c_longlong()
        _check(lib().gpu_mpn_pipe_submit(ctypes.byref(self._c), pz, pa, an, pb, bn, ctypes.byref(t)))
        self._held[t.value] = (a, b, z)
        return t.value

    def wait(self, ticket):
        """The product of `ticket` once it is complete."""
        try:
            _check(lib().gpu_mpn_pipe_wait(ctypes.byref(self._c), ticket))
        finally:
            held = self._held.pop(ticket, None)
        return held[2] if held else None

    def close(self):
        if self._c.impl:
            lib().gpu_mpn_pipe_clear(ctypes.byref(self._c))
            self._c.impl = None
            self._held.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MpnBatch:
    """A planned batch of uneven products on device pointers (gpu_mpn_batch_*).

    `reqs` is a sequence of (z_ptr, a_ptr, an, b_ptr, bn) with device
    pointers as ints.  run() queues every product on `stream` and returns
    without synchronising; check() waits and raises on a kernel error.
    """

    def __init__(self, ctx, reqs, promote_small=0, max_streams=4, use_graph=True, configs=None):
        arr = (MulReq * len(reqs))(*[MulReq(z, a, an, b, bn) for (z, a, an, b, bn) in reqs])
        opt = BatchOptions(promote_small, max_streams, 1 if use_graph else 0)
        cfg = None
        if configs is not None:
            if len(configs) != len(reqs):
                raise ValueError("one configuration per request")
            cfg = (MulConfig * len(reqs))(*[MulConfig(*c.key()) for c in configs])
        self._h = ctypes.c_void_p()
        _check(lib().gpu_mpn_batch_init_config(ctypes.byref(self._h), ctx.ptr, arr, cfg, len(reqs),
                                               ctypes.byref(opt)))

    def run(self, stream=None):
        _check(lib().gpu_mpn_batch_run(self._h, stream))

    def check(self, stream=None):
        _check(lib().gpu_mpn_batch_check(self._h, stream))

    @property
    def launches(self):
        return int(lib().gpu_mpn_batch_launches(self._h))

    @property
    def classes(self):
        return int(lib().gpu_mpn_batch_classes(self._h))

    def close(self):
        if self._h:
            lib().gpu_mpn_batch_clear(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


OP_MUL, OP_SQR, OP_ADDMUL, OP_SUBMUL, OP_ADD, OP_SUB, OP_NEG = range(7)


class Mulmod2expp1:
    """GPU counterpart of sd_fft_mpn_mulmod_2expp1_ctx_t (src/fft_small.h:
    889-923): products modulo 2^N + 1 of (n + 1)-limb operands, N = 64 n."""

    def __init__(self, ctx, N, m=0):
        self.ctx = ctx
        self._c = _Ctx()
        _check(lib().gpu_mulmod_2expp1_ctx_init_status(ctypes.byref(self._c), ctx.ptr, N, m))
        v = [ctypes.c_long() for _ in range(4)]
        _check(lib().gpu_mulmod_2expp1_ctx_info(ctypes.byref(self._c), *[ctypes.byref(x) for x in v]))
        self.N, self.m, self.b, self.np = (x.value for x in v)
        self.n = self.N // 64

    @property
    def ptr(self):
        return ctypes.byref(self._c)

    def mul(self, x, y):
        """z = x y mod 2^N + 1 (host arrays of n + 1 limbs)."""
        x = _limbs(x)
        y = x if y is x else _limbs(y)
        if len(x) != self.n + 1 or len(y) != self.n + 1:
            raise ValueError("operands have n + 1 limbs")
        z = np.zeros(self.n + 1, dtype=np.uint64)
        _check(lib().gpu_mulmod_2expp1_status(self.ptr, z.ctypes.data, x.ctypes.data, y.ctypes.data))
        return z

    def batch_device(self, z_ptr, x_ptr, y_ptr, count, stride=None, stream=None):
        _check(lib().gpu_mulmod_2expp1_batch_device(self.ptr, z_ptr, x_ptr, y_ptr, count,
                                                    stride or self.n + 1, stream))

    def transformed_size(self, count=1):
        return int(lib().gpu_mulmod_2expp1_transformed_size(self.ptr, count))

    def transform_device(self, F_ptr, y_ptr, count, stride=None, stream=None):
        _check(lib().gpu_mulmod_2expp1_transform_device(self.ptr, F_ptr, y_ptr, count,
                                                        stride or self.n + 1, stream))

    def mul_cached_device(self, z_ptr, x_ptr, F_ptr, count, stride=None, stream=None):
        _check(lib().gpu_mulmod_2expp1_mul_cached_device(self.ptr, z_ptr, x_ptr, F_ptr, count,
                                                         stride or self.n + 1, stream))

    def close(self):
        if self._c.impl:
            lib().gpu_mulmod_2expp1_ctx_clear(ctypes.byref(self._c))
            self._c.impl = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MulPrecomp:
    """GPU counterpart of mul_precomp_struct (src/fft_small.h:796-822): b's
    transforms of length 2^depth for modulus n, reused by mul_mid."""

    def __init__(self, ctx, b, depth, n, btrunc=None):
        self.ctx, self.n = ctx, int(n)
        b = _limbs(b)
        self._m = _MulPrecomp()
        _check(lib().gpu_mul_precomp_init_status(ctypes.byref(self._m), b.ctypes.data, len(b),
                                                 btrunc or len(b), depth, _Nmod(self.n, 0, 0), ctx.ptr))
        self.bn, self.depth = len(b), int(self._m.depth)

    @property
    def ptr(self):
        return ctypes.byref(self._m)

    def mul_mid(self, zl, zh, a):
        """Coefficients [zl, zh) of a b mod n, or None when the window does
        not fit the transform (the reference's 0 return)."""
        a = _limbs(a)
        z = np.zeros(max(zh - zl, 0), dtype=np.uint64)
        ok = lib()._gpu_nmod_poly_mul_mid_precomp(z.ctypes.data, zl, zh, a.ctypes.data, len(a), self.ptr,
                                                   _Nmod(self.n, 0, 0), self.ctx.ptr)
        return z if ok else None

    def mul_mid_device(self, z_ptr, zl, zh, a_ptr, an, stream=None):
        _check(lib().gpu_nmod_poly_mul_mid_precomp_device(z_ptr, zl, zh, a_ptr, an, self.ptr, stream))

    def close(self):
        if self._m.impl:
            lib()._gpu_mul_precomp_clear(ctypes.byref(self._m))
            self._m.impl = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DivremPrecomp:
    """GPU counterpart of nmod_poly_divrem_precomp_struct (src/fft_small.h:
    824-848): division by a fixed b with quotients up to Bn coefficients."""

    def __init__(self, ctx, b, Bn, n):
        self.ctx, self.n = ctx, int(n)
        b = _limbs(b)
        self._m = _DivremPrecomp()
        _check(lib()._gpu_nmod_poly_divrem_precomp_init_status(ctypes.byref(self._m), b.ctypes.data, len(b),
                                                              Bn, _Nmod(self.n, 0, 0), ctx.ptr))
        self.bn, self.Bn = len(b), int(Bn)

    @property
    def ptr(self):
        return ctypes.byref(self._m)

    def divrem(self, a):
        """(q, r) with a = q b + r, or None when the quotient is longer than Bn."""
        a = _limbs(a)
        q = np.zeros(len(a) - self.bn + 1, dtype=np.uint64)
        r = np.zeros(self.bn - 1, dtype=np.uint64)
        ok = lib()._gpu_nmod_poly_divrem_precomp(q.ctypes.data, r.ctypes.data, a.ctypes.data, len(a), self.ptr,
                                                 _Nmod(self.n, 0, 0), self.ctx.ptr)
        return (q, r) if ok else None

    def divrem_device(self, q_ptr, r_ptr, a_ptr, an, stream=None):
        _check(lib().gpu_nmod_poly_divrem_precomp_device(q_ptr, r_ptr, a_ptr, an, self.ptr, stream))

    def close(self):
        if self._m.quo_maker.impl or self._m.rem_maker.impl:
            lib()._gpu_nmod_poly_divrem_precomp_clear(ctypes.byref(self._m))
            self._m.quo_maker.impl = self._m.rem_maker.impl = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mulmod_2expp1_choose_np(b, depth):
    return int(lib().gpu_mulmod_2expp1_choose_np(b, depth))


class FftPlan:
    """A plan of the transformed-operand API (gpu_fft_plan_*; the reference's
    fft_small_plan_init_mpn / _nmod).  Build with FftPlan.mpn(...) or
    FftPlan.nmod(...); operands are FftOp objects of the plan."""

    def __init__(self, ctx, handle, kind, mod=None):
        self.ctx, self._h, self.kind, self.mod = ctx, handle, kind, mod
        np_, lm = ctypes.c_int(), ctypes.c_int()
        _check(lib().gpu_fft_plan_info(self._h, ctypes.byref(np_), ctypes.byref(lm)))
        self.np, self.logM = np_.value, lm.value

    @classmethod
    def mpn(cls, ctx, an_max, bn_max, len_bound=None, is_signed=False):
        h = ctypes.c_void_p()
        lb = len_bound if len_bound is not None else min(an_max, bn_max)
        _check(lib().gpu_fft_plan_init_mpn(ctypes.byref(h), ctx.ptr, an_max, bn_max, lb,
                                           1 if is_signed else 0))
        return cls(ctx, h, "mpn")

    @classmethod
    def mpn_np(cls, ctx, an_max, bn_max, len_bound, is_signed, np_):
        h = ctypes.c_void_p()
        _check(lib().gpu_fft_plan_init_mpn_np(ctypes.byref(h), ctx.ptr, an_max, bn_max, len_bound,
                                              1 if is_signed else 0, np_))
        return cls(ctx, h, "mpn")

    @classmethod
    def mpn_cyclic(cls, ctx, nn, len_bound=1):
        """(plan, nn rounded up) for products mod 2^(64 nn) - 1."""
        h = ctypes.c_void_p()
        v = ctypes.c_ulong(nn)
        _check(lib().gpu_fft_plan_init_mpn_cyclic(ctypes.byref(h), ctx.ptr, ctypes.byref(v), len_bound))
        return cls(ctx, h, "mpn"), v.value

    @classmethod
    def nmod_cyclic(cls, ctx, depth, zh, n, len_bound=None, prod_bits=None):
        h = ctypes.c_void_p()
        pb = prod_bits if prod_bits is not None else 2 * (int(n) - 1).bit_length()
        _check(lib().gpu_fft_plan_init_nmod_cyclic(ctypes.byref(h), ctx.ptr, depth, zh,
                                                   len_bound or (1 << depth), pb, _Nmod(n, 0, 0)))
        return cls(ctx, h, "nmod", n)

    def sizeof_data(self):
        return int(lib().gpu_fft_op_sizeof_data(self._h))

    @classmethod
    def nmod(cls, ctx, zl, zh, zn, n, len_bound, prod_bits=None):
        h = ctypes.c_void_p()
        pb = prod_bits if prod_bits is not None else 2 * (int(n) - 1).bit_length()
        _check(lib().gpu_fft_plan_init_nmod(ctypes.byref(h), ctx.ptr, zl, zh, zn, len_bound, pb,
                                            _Nmod(n, 0, 0)))
        return cls(ctx, h, "nmod", n)

    def op(self, data_ptr=None):
        """A transformed operand; with data_ptr, in that caller-owned device
        memory (sizeof_data() bytes)."""
        return FftOp(self, data_ptr)

    def pointwise(self, op, Z, A, B=None, stream=None):
        _check(lib().gpu_fft_op_pointwise(op, Z._h, A._h, (B or A)._h, self._h, stream))

    def check(self, stream=None):
        _check(lib().gpu_fft_op_check(self._h, stream))

    def close(self):
        if self._h:
            lib().gpu_fft_plan_clear(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FftOp:
    """A transformed operand (gpu_fft_op_*), resident in device memory."""

    def __init__(self, plan, data_ptr=None):
        self.plan = plan
        self._h = ctypes.c_void_p()
        if data_ptr is None:
            _check(lib().gpu_fft_op_init(ctypes.byref(self._h), plan._h))
        else:
            _check(lib().gpu_fft_op_init_borrowed(ctypes.byref(self._h), plan._h, data_ptr))

    def fft(self, a_ptr, an, stream=None):
        f = lib().gpu_fft_fft_mpn if self.plan.kind == "mpn" else lib().gpu_fft_fft_nmod
        _check(f(self._h, a_ptr, an, self.plan._h, stream))

    def ifft(self, stream=None):
        _check(lib().gpu_fft_ifft(self._h, self.plan._h, stream))

    def export_mpn(self, z_ptr, zn, stream=None):
        _check(lib().gpu_fft_export_mpn(z_ptr, zn, self._h, self.plan._h, stream))

    def export_mpn_signed(self, z_ptr, zn, nslots, lo_limbs=0, stream=None):
        """Limbs [lo_limbs, lo_limbs + zn) of |value| into z; returns the sign
        (1 negative).  Synchronises the stream."""
        sg = ctypes.c_int()
        _check(lib().gpu_fft_export_mpn_signed_trunc(z_ptr, zn, ctypes.byref(sg), self._h, nslots, lo_limbs,
                                                     self.plan._h, stream))
        return sg.value

    def export_nmod(self, z_ptr, zl, zh, stream=None):
        _check(lib().gpu_fft_export_nmod(z_ptr, zl, zh, self._h, _Nmod(self.plan.mod, 0, 0),
                                         self.plan._h, stream))

    def close(self):
        if self._h:
            lib().gpu_fft_op_clear(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
