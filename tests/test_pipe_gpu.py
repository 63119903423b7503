"""GPU parity of pipelined host-pointer products (gpu_mpn_pipe_*).

Every product that goes through a pipeline must equal GMP's mpn_mul limb for
limb, whatever the interleaving of submissions and waits: products of mixed
sizes sharing slots, squarings, pinned and pageable host buffers, the full
2^24 x 2^24 size, and the ticket rules (every ticket is waited for once, in
any order; unknown tickets and second waits are errors, and the pipeline
stays usable after them).
"""
import numpy as np
import pytest

import flint_b200 as FB
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_mixed_sizes_in_submission_order(depth):
    sizes = [(5000, 3000), (1, 1), (70000, 65000), (300000, 5000), (17, 16), (131072, 131072),
             (4096, 1), (65537, 65535)]
    ops = [(O.rand_limbs(40 + k, an), O.rand_limbs(80 + k, bn)) for k, (an, bn) in enumerate(sizes)]
    with FB.MpnPipe(depth) as P:
        tickets = [P.submit(a, b) for a, b in ops]
        for t, (a, b) in zip(tickets, ops):
            assert (P.wait(t) == O.gmp_mpn_mul(a, b)).all()


def test_waits_interleaved_with_submissions():
    """Each wait right after the submission that reuses its slot; squarings."""
    with FB.MpnPipe(2) as P:
        pend = []
        for k in range(7):
            a = O.rand_limbs(200 + k, 20000 + 1000 * k)
            b = a if k % 3 == 0 else O.rand_limbs(300 + k, 9000 + 777 * k)
            pend.append((P.submit(a, b), a, b))
            if len(pend) == 2:
                t, a0, b0 = pend.pop(0)
                assert (P.wait(t) == O.gmp_mpn_mul(a0, b0)).all()
        for t, a0, b0 in pend:
            assert (P.wait(t) == O.gmp_mpn_mul(a0, b0)).all()


def test_pinned_tensors_full_size():
    torch = pytest.importorskip("torch")
    n = 1 << 24
    ops = [(O.rand_limbs(7, n), O.rand_limbs(8, n)), (O.rand_limbs(9, n), O.rand_limbs(10, n - 4321))]
    pinned = [(torch.from_numpy(a.view(np.int64)).pin_memory(), torch.from_numpy(b.view(np.int64)).pin_memory(),
               torch.empty(len(a) + len(b), dtype=torch.int64).pin_memory()) for a, b in ops]
    with FB.MpnPipe(2) as P:
        tickets = [P.submit(ha, hb, out=hz) for ha, hb, hz in pinned]
        for t, (a, b), (_, _, hz) in zip(tickets, ops, pinned):
            P.wait(t)
            assert (hz.numpy().view(np.uint64) == O.gmp_mpn_mul(a, b)).all()


def test_ticket_rules():
    with FB.MpnPipe(2) as P:
        a, b = O.rand_limbs(1, 3000), O.rand_limbs(2, 2000)
        want = O.gmp_mpn_mul(a, b)
        t0 = P.submit(a, b)
        t1 = P.submit(a, b)
        t2 = P.submit(a, b)            # completes t0 (same slot)
        t3 = P.submit(a, b)            # completes t1
        assert (P.wait(t2) == want).all()
        assert (P.wait(t0) == want).all()   # completed earlier, waited later
        with pytest.raises(FB.GpuFftSmallError) as e:
            P.wait(t0)                  # second wait
        assert e.value.code == FB.EINVAL
        assert (P.wait(t3) == want).all()
        with pytest.raises(FB.GpuFftSmallError) as e:
            P.wait(99)                  # never submitted
        assert e.value.code == FB.EINVAL
        assert (P.wait(t1) == want).all()
        with pytest.raises(FB.GpuFftSmallError) as e:
            P.submit(np.zeros(0, np.uint64), b)
        assert e.value.code == FB.EINVAL
        # still usable
        t4 = P.submit(b, a)
        assert (P.wait(t4) == O.gmp_mpn_mul(b, a)).all()


def test_close_completes_products_in_flight():
    a, b = O.rand_limbs(11, 50000), O.rand_limbs(12, 40000)
    z = np.zeros(90000, dtype=np.uint64)
    P = FB.MpnPipe(3)
    P.submit(a, b, out=z)
    P.close()                           # waits for the product before freeing the slots
    assert (z == O.gmp_mpn_mul(a, b)).all()
