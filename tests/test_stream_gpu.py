"""The request-stream executor under a schedule: every product identical to
the product under the fixed rule, and a subsample identical to the
reference's own products."""
import numpy as np
import pytest

import oracle as O
from flint_b200 import tuner
from flint_b200.stream import run_stream
from flint_b200.workload import request_stream

pytestmark = pytest.mark.gpu


def test_stream_schedules_agree_and_match_reference(ctx):
    torch = pytest.importorskip("torch")
    reqs = request_stream(31, 40, mpn_log=(0.0, 17.0), fmpz_len_log=(4.0, 10.0),
                          fmpz_bits=(64, 700))
    # a deliberately varied schedule: cycle through each request's candidates
    cfgs = [tuner.candidates(r)[k % len(tuner.candidates(r))] for k, r in enumerate(reqs)]
    default = [tuner.default_config(r) for r in reqs]
    stream = torch.cuda.current_stream()
    keep = set(range(0, 40, 3))
    res = run_stream(ctx, torch, reqs, cfgs, 5, stream, torch.device("cuda"), chunk_limbs=1 << 18,
                     keep=keep, check_against=default)
    assert res["identical"]
    assert res["mpn_requests"] + res["fmpz_requests"] == len(reqs)
    for k in keep:
        r = reqs[k]
        if r[0] == 0:
            ops, z = res["kept"][k]
            an, bn = r[1], r[2]
            assert (z == O.gmp_mpn_mul(ops[:an], ops[an:an + bn])).all()
        else:
            a, b, z = res["kept"][k]
            _, an, bn, aw, bw = r
            want = O.fmpz_poly_mul_python(O.raw_to_ints(a.reshape(an, aw)),
                                          O.raw_to_ints(b.reshape(bn, bw)))
            assert O.raw_to_ints(z.reshape(an + bn - 1, aw + bw + 1)) == want
