"""GPU parity of integer-polynomial products (_fmpz_poly_mul_mid_mpn_ctx).

Every coefficient is compared exactly: against the Python Kronecker
restatement at small sizes, against the reference's own _fmpz_poly_mul
(src/fmpz_poly/mul.c:100-186) through the compiled reference library, and --
at the largest request-stream size (2^16 x 2^16 coefficients of 4096 bits) --
against the reference plus an evaluation fingerprint.  Edge cases follow the
reference's test (src/fft_small/test/t-fmpz_poly_mul.c): signed coefficients,
unequal lengths and widths, squaring, windows that start late or run past
the product, zero polynomials.
"""
import ctypes

import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not O.have_ref(), reason="reference library not built")


def _gpu_ints(ctx, a_raw, b_raw, zl=0, zh=None):
    zh = len(a_raw) + len(b_raw) - 1 if zh is None else zh
    return O.raw_to_ints(ctx.fmpz_poly_mul_mid(zl, zh, a_raw, b_raw))


@pytest.mark.parametrize("an,bn,ba,bb", [
    (1, 1, 1, 1), (1, 5, 63, 64), (7, 3, 64, 65), (40, 33, 100, 20), (256, 256, 64, 64),
    (300, 17, 500, 9), (1000, 999, 130, 130), (5, 2000, 2000, 70), (4096, 4096, 63, 62),
])
def test_vs_python(ctx, an, bn, ba, bb):
    a = O.rand_fmpz_raw(an * 31 + ba, an, ba)
    b = O.rand_fmpz_raw(bn * 17 + bb, bn, bb)
    want = O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(b))
    assert _gpu_ints(ctx, a, b) == want


@pytest.mark.parametrize("an,bn,ba,bb", [
    (40, 30, 250, 300),              # slot stride S = 4 + 5 - 1 = 8: one thread per coefficient
    (40, 30, 300, 300),              # S = 9: the tiled CRT, 227 coefficients per block
    (3, 2, 65535, 65536),            # S = 1024 + 1025 - 1 = 2048: tiled, one coefficient per block
    (3, 2, 65536, 65536),            # S = 2049: one thread per coefficient again
])
def test_crt_layout_boundaries(ctx, an, bn, ba, bb):
    """Both integer-polynomial CRT kernels at the slot strides where the
    library switches between them, whole products and windows that start
    and end inside a block's run of coefficients."""
    a = O.rand_fmpz_raw(an + ba, an, ba)
    b = O.rand_fmpz_raw(bn + 3 * bb, bn, bb)
    full = O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(b))
    zn = len(full)
    assert _gpu_ints(ctx, a, b) == full
    for zl, zh in [(1, zn), (zn // 2, zn - 1), (zn - 1, zn + 2)]:
        want = [full[k] if k < zn else 0 for k in range(zl, zh)]
        assert _gpu_ints(ctx, a, b, zl, zh) == want, (zl, zh)


def test_crt_tiled_many_blocks(ctx):
    """The tiled CRT over many blocks (S = 9, 227 coefficients each), with
    windows that start and end mid-block, and a squaring."""
    a = O.rand_fmpz_raw(77, 400, 300)
    b = O.rand_fmpz_raw(78, 350, 290)
    full = O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(b))
    zn = len(full)
    for zl, zh in [(0, zn), (5, 460), (226, 229), (227, 681), (zn - 300, zn + 10)]:
        want = [full[k] if k < zn else 0 for k in range(zl, zh)]
        assert _gpu_ints(ctx, a, b, zl, zh) == want, (zl, zh)
    assert _gpu_ints(ctx, a, a) == O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(a))


def test_windows_and_zero_fill(ctx):
    a = O.rand_fmpz_raw(1, 50, 90)
    b = O.rand_fmpz_raw(2, 30, 200)
    full = O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(b))
    zn = len(full)
    for zl, zh in [(0, 1), (10, 20), (zn - 1, zn), (zn - 5, zn + 7), (zn, zn + 3), (3, 3)]:
        got = _gpu_ints(ctx, a, b, zl, zh)
        want = [full[k] if k < zn else 0 for k in range(zl, zh)]
        assert got == want, (zl, zh)


def test_squaring_and_extremes(ctx):
    a = O.rand_fmpz_raw(9, 777, 300)
    want = O.fmpz_poly_mul_python(O.raw_to_ints(a), O.raw_to_ints(a))
    assert _gpu_ints(ctx, a, a) == want
    # extreme magnitudes: +-(2^B - 1) everywhere, and a zero polynomial
    B = 256
    vals = [((1 << B) - 1) * (1 if k % 3 else -1) for k in range(200)]
    r = O.ints_to_raw(vals, 5)
    assert _gpu_ints(ctx, r, r) == O.fmpz_poly_mul_python(vals, vals)
    zero = np.zeros((10, 1), dtype=np.uint64)
    assert _gpu_ints(ctx, zero, r) == [0] * 209
    # wider rows than needed (sign extension) give the same product
    a2 = O.ints_to_raw(O.raw_to_ints(a), 9)
    assert _gpu_ints(ctx, a2, a) == want


@needs_ref
@pytest.mark.parametrize("an,bn,ba,bb", [(3000, 2500, 64, 64), (2048, 100, 1000, 4096),
                                         (700, 700, 3000, 3000)])
def test_vs_reference(ctx, an, bn, ba, bb):
    a = O.rand_fmpz_raw(an + 3 * ba, an, ba)
    b = O.rand_fmpz_raw(bn + 5 * bb, bn, bb)
    zw = FB.fmpz_result_width(a, b)
    want = O.ref_fmpz_poly_mul_raw(a, b, zw)
    got = ctx.fmpz_poly_mul_mid(0, an + bn - 1, a, b, zw)
    assert (got == want).all()


@needs_ref
def test_largest_request_size_vs_reference(ctx):
    """2^16 x 2^16 coefficients of 4096 bits: a 2^25-point chunk product."""
    n, B = 1 << 16, 4096
    a = O.rand_fmpz_raw(101, n, B)
    b = O.rand_fmpz_raw(102, n, B)
    zw = (2 * B + 16 + 1 + 63) // 64
    got = ctx.fmpz_poly_mul_mid(0, 2 * n - 1, a, b, zw)
    want = O.ref_fmpz_poly_mul_raw(a, b, zw)
    assert (got == want).all()
    # evaluation fingerprint at x0 mod a 61-bit prime
    q, x0 = 2305843009213693951, 123456789

    def ev(raw):
        vals = [v % q for v in O.raw_to_ints(raw)]
        acc = 0
        for v in reversed(vals):
            acc = (acc * x0 + v) % q
        return acc
    assert ev(got) == ev(a) * ev(b) % q


@needs_ref
def test_fmpz_drop_in_with_reference_vectors(ctx):
    """The fmpz entry point on vectors the reference allocated (inline values
    and mpz pointers mixed), output through fmpz_set_signed_ui_array, compared
    with the reference's own product by _fmpz_vec_equal."""
    L = O._ref_fmpz()
    lib = FB.lib()
    hook = ctypes.cast(L.fmpz_set_signed_ui_array, ctypes.c_void_p).value
    lib.gpu_fmpz_set_signed_hook(hook)
    try:
        for (an, bn, ba, bb) in [(500, 300, 40, 2000), (64, 64, 61, 62), (1000, 1000, 200, 10)]:
            a = O.rand_fmpz_raw(an + 1, an, ba)
            b = O.rand_fmpz_raw(bn + 2, bn, bb)
            zn = an + bn - 1
            with O.RefFmpzVec(an) as A, O.RefFmpzVec(bn) as Bv, O.RefFmpzVec(zn) as Z, \
                    O.RefFmpzVec(zn) as W:
                A.set_raw(a)
                Bv.set_raw(b)
                hi, lo = (A, Bv) if an >= bn else (Bv, A)
                L._fmpz_poly_mul(W.ptr, hi.ptr, max(an, bn), lo.ptr, min(an, bn))
                rc = lib._gpu_fmpz_poly_mul_mid_mpn_ctx(Z.ptr, 0, zn, A.ptr, an, Bv.ptr, bn, ctx.ptr)
                assert rc == 1
                assert L._fmpz_vec_equal(Z.ptr, W.ptr, zn) == 1
    finally:
        lib.gpu_fmpz_set_signed_hook(None)


def test_fmpz_inline_values_without_hook(ctx):
    """Without a setter the fmpz entry point handles inline results only."""
    lib = FB.lib()
    a = (ctypes.c_long * 4)(3, -7, 1 << 20, -(1 << 25))
    b = (ctypes.c_long * 3)(-2, 5, 1 << 10)
    z = (ctypes.c_long * 7)(*([99] * 7))
    assert lib._gpu_fmpz_poly_mul_mid_mpn_ctx(z, 0, 7, a, 4, b, 3, ctx.ptr) == 1
    want = O.fmpz_poly_mul_python(list(a), list(b)) + [0]
    assert list(z) == want


def test_device_entry_point(ctx):
    torch = pytest.importorskip("torch")
    a = O.rand_fmpz_raw(41, 3000, 150)
    b = O.rand_fmpz_raw(42, 2000, 70)
    zw = FB.fmpz_result_width(a, b)
    zn = 4999
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.full((zn + 5, zw), -1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    ctx.fmpz_poly_mul_device(dz.data_ptr(), zw, 0, zn + 5, da.data_ptr(), a.shape[1], 3000,
                             db.data_ptr(), b.shape[1], 2000, stream.cuda_stream)
    stream.synchronize()
    got = dz.cpu().numpy().view(np.uint64)
    assert (got == ctx.fmpz_poly_mul_mid(0, zn + 5, a, b, zw)).all()
    assert not got[zn:].any()


@pytest.mark.parametrize("name", ["fmpz_1x1", "fmpz_40x33_signed", "fmpz_300x17_wide",
                                  "fmpz_1000x999_130", "fmpz_2048x100_1000x4096",
                                  "fmpz_square_777_300", "fmpz_window_500x400",
                                  "fmpz_2^16x2^16_4096"])
def test_golden_fmpz(ctx, golden, name):
    from tests.golden.make_golden import fmpz_inputs
    case = next(c for c in golden["fmpz"] if c["name"] == name)
    a, b, zw, zl, zh = fmpz_inputs(case)
    flat = ctx.fmpz_poly_mul_mid(zl, zh, a, b, zw).reshape(-1)
    if "full" in case:
        assert ["%016x" % int(v) for v in flat] == case["full"]
    else:
        assert O.digest(flat) == case["digest"] and len(flat) == case["len"]


@pytest.mark.parametrize("an,bn,aw,bw,sq", [
    (4500, 4500, 32, 32, False),      # 8999 x 63 positions: 3 2^18 points instead of 2^20
    (9000, 5000, 20, 20, False),      # 13999 x 39: 3 2^18
    (17000, 17000, 32, 32, False),    # 33999 x 63: 3 2^20 instead of 2^22
    (4500, 4500, 32, 32, True),       # a squaring on 3 2^18 points
])
def test_three_length_equals_power_of_two(ctx, an, bn, aw, bw, sq):
    """Integer-polynomial products on 3 2^k-point transforms (the default
    without a configuration, and the THREE flag) equal the same products on
    the power-of-two transform, coefficient for coefficient; the largest
    request-size test checks the 3 2^23-point case against the reference."""
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cuda")
    g.manual_seed(an + 3 * bn + aw)
    a = torch.randint(-(1 << 63), (1 << 63) - 1, (an * aw,), dtype=torch.int64, device="cuda", generator=g)
    b = a if sq else torch.randint(-(1 << 63), (1 << 63) - 1, (bn * bw,), dtype=torch.int64, device="cuda",
                                   generator=g)
    if sq:
        bn, bw = an, aw
    zw, zn = aw + bw + 1, an + bn - 1
    plain = FB.resolve_config(1, an, bn, None, aw, bw)
    assert plain.flags == 0
    three = FB.resolve_config(1, an, bn, FB.MulConfig(FB.ROUTE_NTT, 0, 0, 0, FB.FLAG_THREE), aw, bw)
    assert three.logM == plain.logM and three.logC == 13
    s = torch.cuda.current_stream()
    outs = []
    for cfg in (plain, three, None):
        z = torch.full((zn * zw,), -1, dtype=torch.int64, device="cuda")
        if cfg is None:
            ctx.fmpz_poly_mul_device(z.data_ptr(), zw, 0, zn, a.data_ptr(), aw, an, b.data_ptr(), bw, bn,
                                     s.cuda_stream)
        else:
            ctx.fmpz_poly_mul_device_config(z.data_ptr(), zw, 0, zn, a.data_ptr(), aw, an, b.data_ptr(), bw,
                                            bn, cfg, s.cuda_stream)
        s.synchronize()
        outs.append(z.cpu())
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
