"""The hand-written backward seen from torch (test harness only).

A torch.autograd.Function whose forward runs nrrs_train_grads on the GPU (the library's forward,
both losses and its hand-written backward, without the Adam update) and whose backward returns
the library's parameter gradients. The gradients that torch then produces are checked against
the FP64 oracle's gradient and against central finite differences of the GPU's own losses.

The two losses train disjoint parameter sets. The StatNet loss trains the hash table and
StatNet; the RRSNet loss trains RRSNet, on inputs taken from a detached StatNet forward, as in
the reference (network.cpp:196-295). So the Function returns both losses, and each parameter's
gradient is that of the loss which trains it.
"""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu


def _function():
    torch = torch_cuda()

    class NRRSTrainLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, net, batch, n):
            net.set_params(params.detach().cpu().numpy().astype(np.float32))
            loss = torch.zeros(2, dtype=torch.float64, device="cuda")
            net.trainGrads(soa(batch), batch["target"], n, loss, stream())
            torch.cuda.synchronize()
            g = torch.from_numpy(net.get_grads().astype(np.float64))
            ctx.save_for_backward(g)
            ctx.layout = net.param_layout()
            return loss.cpu()

        @staticmethod
        def backward(ctx, grad_loss):
            (g,) = ctx.saved_tensors
            ntab, nst, _ = ctx.layout
            out = g.clone()
            out[:ntab + nst] *= grad_loss[0]      # table and StatNet: StatNet loss
            out[ntab + nst:] *= grad_loss[1]      # RRSNet: RRSNet loss
            return out, None, None, None

    return NRRSTrainLoss


def _setup(seed=71, n=4096):
    net = make_net(max_train=1 << 13, step=3, log2_hashmap_size=15)
    p0 = random_params(net, seed, table_scale=0.5, mlp_scale=0.15)
    v = nb.synth(seed + 1, n)
    return net, p0, v, upload(v), n


def test_autograd_gradient_matches_fp64_oracle():
    torch = torch_cuda()
    fn = _function()
    net, p0, v, batch, n = _setup()
    params = torch.tensor(p0.astype(np.float64), requires_grad=True)
    loss = fn.apply(params, net, batch, n)
    loss.sum().backward(retain_graph=True)
    g = params.grad.numpy().copy()
    g64, l64 = O.train_grads(net.config, p0, v, v["target"], "f64")
    assert loss.detach().numpy() == pytest.approx(l64, rel=1e-5)
    ntab, nst, nrr = net.param_layout()
    for sl in (slice(0, ntab), slice(ntab, ntab + nst), slice(ntab + nst, ntab + nst + nrr)):
        e = np.linalg.norm(g[sl] - g64[sl]) / np.linalg.norm(g64[sl])
        assert e < 2e-4, (sl, e)
    # a weighted objective scales each group by its loss weight
    params.grad = None
    (2.0 * loss[0] + 0.5 * loss[1]).backward()
    g2 = params.grad.numpy()
    assert np.allclose(g2[:ntab + nst], 2.0 * g[:ntab + nst])
    assert np.allclose(g2[ntab + nst:], 0.5 * g[ntab + nst:])
    net.close()


def test_autograd_gradient_matches_gpu_finite_differences():
    """central differences of the GPU's FP32-forward losses (h = 1e-3, as the FP64 oracle test
    uses) on the 12 largest-gradient parameters of each group; the losses are FP64 sums of
    FP32 per-sample terms, so the bar is 3e-2 relative"""
    torch = torch_cuda()
    fn = _function()
    net, p0, v, batch, n = _setup(seed=73)
    params = torch.tensor(p0.astype(np.float64), requires_grad=True)
    loss = fn.apply(params, net, batch, n)
    loss.sum().backward()
    g = params.grad.numpy()
    ntab, nst, nrr = net.param_layout()
    h = 1e-3
    worst = {}
    for name, lo, hi, which in (("table", 0, ntab, 0), ("statnet", ntab, ntab + nst, 0),
                                ("rrsnet", ntab + nst, ntab + nst + nrr, 1)):
        idx = lo + np.argsort(-np.abs(g[lo:hi]))[:12]
        errs = []
        for k in idx:
            pp = p0.astype(np.float64).copy()
            pp[k] += h
            lp = fn.apply(torch.tensor(pp), net, batch, n)[which].item()
            pp[k] -= 2 * h
            lm = fn.apply(torch.tensor(pp), net, batch, n)[which].item()
            fd = (lp - lm) / (2 * h)
            errs.append(abs(fd - g[k]) / max(abs(g[k]), 1e-12))
        worst[name] = max(errs)
    for name, e in worst.items():
        assert e < 3e-2, (name, e, worst)
    net.close()
