"""GPU test of nrrs_decide_emit_noalloc, the decision + emission entry point that allocates no
device memory (for callers that cannot call cudaMalloc: plugins whose host framework owns all
device memory, fixed start-up memory budgets, frame loops that must not synchronise).

Its results must equal those of nrrs_decide_emit on a context whose max_queue is
NRRS_NOALLOC_MAX_N (same exact-sum shift), bit for bit, on two calls in a row: the second call
checks that the static scratch left behind by the first does not leak into its result. This
file is collected last so a failure here cannot hide the other tests' results."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
from gpu_util import empty, host, make_net, stream, torch_cuda

pytestmark = pytest.mark.gpu


def _inputs(seed, n):
    rng = np.random.default_rng(seed)
    rrs = np.clip(rng.lognormal(-0.2, 1.1, n), 0.05, 8).astype(np.float32)
    rnd = rng.random(n, dtype=np.float32)
    return rrs, rnd


def _outputs(n, cap):
    return dict(norm=empty(n), split=empty(n, "uint8"), q=empty(cap, "int32"), sz=empty(1, "int32"))


def _host(o, n):
    tot = int(host(o["sz"], np.uint32)[0])
    return {"total": tot, "queue": host(o["q"], np.uint32)[:tot].copy(),
            "split": host(o["split"])[:n].copy(), "norm": host(o["norm"])[:n].view(np.uint32).copy()}


def test_noalloc_matches_context_entry_point_twice():
    torch = torch_cuda()
    net = make_net(max_queue=nb.NOALLOC_MAX_N, max_train=1024)
    s = stream()
    for call, (seed, n, use_ceil) in enumerate([(11, 300_007, 1), (12, 1_000_003, 0)]):
        rrs, rnd = _inputs(seed, n)
        d_rrs, d_rnd = torch.from_numpy(rrs).cuda(), torch.from_numpy(rnd).cuda()
        dp = nb.default_decide(use_ceil=use_ceil)
        cap = 9 * n
        ref, got = _outputs(n, cap), _outputs(n, cap)
        net.decideEmit(d_rrs, d_rnd, n, n, n // 40, dp, ref["norm"], ref["split"], ref["q"], cap,
                       ref["sz"], stream=s)
        rc = nb.decide_emit_noalloc(d_rrs, d_rnd, n, n, n // 40, dp, got["norm"], got["split"],
                                    got["q"], cap, got["sz"], stream=s)
        assert rc == nb.OK, (call, rc)
        torch.cuda.synchronize()
        a, b = _host(ref, n), _host(got, n)
        assert a["total"] == b["total"] > 0, call
        assert np.array_equal(a["queue"], b["queue"]), call
        assert np.array_equal(a["split"], b["split"]), call
        assert np.array_equal(a["norm"], b["norm"]), call
    net.close()


def test_noalloc_rejects_oversize_and_handles_empty():
    torch = torch_cuda()
    dp = nb.default_decide()
    o = _outputs(1, 1)
    rc = nb.decide_emit_noalloc(empty(1), empty(1), nb.NOALLOC_MAX_N + 1, 10, 0, dp, o["norm"],
                                o["split"], o["q"], 1, o["sz"], stream=stream())
    assert rc == nb.ERR_INVALID_ARG
    o["sz"].fill_(7)
    rc = nb.decide_emit_noalloc(empty(1), empty(1), 0, 10, 0, dp, o["norm"], o["split"], o["q"],
                                1, o["sz"], stream=stream())
    torch.cuda.synchronize()
    assert rc == nb.OK and int(host(o["sz"], np.uint32)[0]) == 0
