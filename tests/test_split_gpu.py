"""GPU parity of split products: an unbalanced whole product whose long
operand is cut into chunks, each multiplied by the short one in a shorter
transform, the chunks' residues summed into one array of the full length and
recombined by a single CRT/carry pass.  Every case is compared limb for limb
with GMP's mpn_mul; the sizes cover several chunk lengths (2^20 to 2^23
points), short last chunks, a one-limb short operand (no overlap between
chunks), the operands in either order, and products for which splitting
does not pay (they take the single transform).
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu

C20 = (1 << 20) - 3000 + 1    # chunk length of 2^20-point chunks against 3000 limbs

SIZES = [
    (1 << 24, 1 << 20),            # 6 chunks of 2^22 points
    (1 << 22, 3000),               # 5 chunks of 2^20 points
    (3000, 1 << 22),               # the same with the operands swapped
    (5 * C20 + 1, 3000),           # 3 chunks of 2^21 points
    ((1 << 23) + (1 << 20), 1),    # one-limb short operand: 5 chunks that do not overlap
    (5_000_000, 300_000),          # 3 chunks of 2^21 points
    (1 << 23, 700_000),            # 3 chunks of 2^22 points
    (1 << 21, 1 << 17),            # not split
    (1 << 24, 1 << 22),            # 4 chunks of 2^23 points
    ((1 << 23), 1),                # not split: eight 2^20-point chunks cost more
    (3 << 20, 1 << 16),            # not split
    ((1 << 22) - (1 << 20), 1 << 20),  # not split
]


@pytest.mark.parametrize("an,bn", SIZES)
def test_split_product_vs_gmp(ctx, an, bn):
    a = O.rand_limbs(an % 997 + 1, an)
    b = O.rand_limbs(bn % 991 + 2, bn)
    assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


def test_split_product_all_ones_and_device_entry(ctx):
    """Longest carry chains across chunk boundaries, through the
    device-pointer entry point."""
    torch = pytest.importorskip("torch")
    an, bn = 5 * C20 + 17, 3000          # 3 chunks of 2^21 points
    ones = np.full(an, (1 << 64) - 1, dtype=np.uint64)
    b = np.full(bn, (1 << 64) - 1, dtype=np.uint64)
    da = torch.from_numpy(ones.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    dz = torch.empty(an + bn, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    ctx.mpn_mul_device(dz.data_ptr(), da.data_ptr(), an, db.data_ptr(), bn, s.cuda_stream)
    s.synchronize()
    assert (dz.cpu().numpy().view(np.uint64) == O.gmp_mpn_mul(ones, b)).all()


@pytest.mark.parametrize("an,bn", [((1 << 25) + (1 << 20), 1000), ((1 << 26) + 12345, 4096)])
def test_products_beyond_the_longest_transform(ctx, an, bn):
    """More than 2^25 + 1 limbs in all: no single transform holds the
    product, chunks of the long operand do."""
    a = O.rand_limbs(an % 1009 + 1, an)
    b = O.rand_limbs(bn % 1013 + 3, bn)
    assert FB.mpn_mul_split_plan(an, bn) > 0
    assert (ctx.mpn_mul(a, b) == O.gmp_mpn_mul(a, b)).all()


def test_split_product_through_the_pipeline():
    a, b = O.rand_limbs(5, 1 << 22), O.rand_limbs(6, 3000)
    with FB.MpnPipe(2) as P:
        t = [P.submit(a, b), P.submit(b, a)]
        want = O.gmp_mpn_mul(a, b)
        assert (P.wait(t[0]) == want).all()
        assert (P.wait(t[1]) == want).all()
