"""The moving average of the weights (nrrs_config.ema_decay; the Ema optimizer that wraps Adam in
common/configs/nrrs/nrrs/2net-simple.json:17-20, decay 0.95): after every Adam step
e <- d e + (1 - d) w, and inference uses e / (1 - d^t) while training keeps using w.

Checked against a float32 restatement of that update on the trained weights read back after each
step (bit for bit), and through inference: a context with the moving average infers exactly what
a context without one infers after uploading the restated average."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
from gpu_util import empty, host, make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu


def _ema_restated(ws, d):
    """float32: e_t = d e_{t-1} + (1 - d) w_t (each product and the sum rounded), e_0 = 0;
    returns e_T / (1 - d^T) with the reciprocal rounded to float32 once"""
    d32 = np.float32(d)
    omd = np.float32(1.0) - d32
    e = np.zeros_like(ws[0])
    for w in ws:
        e = (d32 * e) + (omd * w)
    inv = np.float32(1.0 / (1.0 - float(d32) ** len(ws)))
    return e * inv


def _infer(net, d, n, dp):
    torch = torch_cuda()
    st, rr = empty(6 * n), empty(n)
    net.inference(soa(d), n, dp, st, rr, stream())
    torch.cuda.synchronize()
    return host(st)[:6 * n].copy(), host(rr)[:n].copy()


@pytest.mark.parametrize("prec", [nb.PREC_FP32, nb.PREC_FP16], ids=["fp32", "fp16"])
@pytest.mark.parametrize("family", ["workload", "reference"])
def test_moving_average_matches_restatement_and_drives_inference(prec, family):
    torch = torch_cuda()
    d = 0.95
    kw = dict(precision=prec, max_queue=1 << 16, max_train=1 << 13, log2_hashmap_size=16,
              ema_decay=d)
    if family == "reference":
        cfg = nb.reference_config(**kw)
    else:
        cfg = nb.default_config(step=3, **kw)
    net = nb.NRRSNetwork(cfg)
    random_params(net, 97, table_scale=0.5, mlp_scale=0.15)
    assert np.array_equal(net.get_inference_params(), net.get_params())
    n = 6000
    v = nb.synth(98, n)
    dv = upload(v)
    trained = []
    for _ in range(4):
        loss = torch.zeros(2, dtype=torch.float64, device="cuda")
        net.train(soa(dv), dv["target"], n, loss, stream())
        torch.cuda.synchronize()
        trained.append(net.get_params())
    pinf = net.get_inference_params()
    want = _ema_restated(trained, d)
    assert np.array_equal(pinf, want)
    assert not np.array_equal(pinf, trained[-1])

    # inference runs on the average: equal to a context without one holding those weights
    dp = nb.default_decide()
    st_a, rr_a = _infer(net, dv, n, dp)
    twin_kw = dict(kw, ema_decay=0.0)
    twin = nb.NRRSNetwork(nb.reference_config(**twin_kw) if family == "reference"
                          else nb.default_config(step=3, **twin_kw))
    twin.set_params(want)
    st_b, rr_b = _infer(twin, dv, n, dp)
    assert np.array_equal(rr_a, rr_b)
    assert np.array_equal(st_a, st_b)
    twin.close()

    # training keeps using the trained weights: the losses of a gradient pass equal those of a
    # context holding the trained weights
    twin2 = nb.NRRSNetwork(nb.reference_config(**twin_kw) if family == "reference"
                           else nb.default_config(step=3, **twin_kw))
    twin2.set_params(trained[-1])
    la = torch.zeros(2, dtype=torch.float64, device="cuda")
    lb = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainGrads(soa(dv), dv["target"], n, la, stream())
    twin2.trainGrads(soa(dv), dv["target"], n, lb, stream())
    torch.cuda.synchronize()
    assert torch.equal(la, lb)
    twin2.close()

    # an upload restarts the average
    net.set_params(trained[0])
    assert np.array_equal(net.get_inference_params(), trained[0])
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


def test_ema_decay_out_of_range_is_rejected():
    for bad in (-0.1, 1.0, float("nan")):
        with pytest.raises(nb.NRRSError):
            make_net(max_queue=1 << 10, max_train=1 << 10, log2_hashmap_size=12, ema_decay=bad)
