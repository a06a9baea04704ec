"""GPU parity of the training step (nrrs_train_step) against the oracle: losses, gradients of
the hash table and both MLPs before the update, and the Adam update itself."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import empty, host, make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu


def run_step(net, v, n):
    torch = torch_cuda()
    d = upload(v)
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.train(soa(d), d["target"], n, loss, stream())
    torch.cuda.synchronize()
    return loss.cpu().numpy()


def rel_err(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("step", [3, 2])
def test_fp32_grads_and_losses_vs_fp64_oracle(step):
    net = make_net(max_train=1 << 14, step=step, log2_hashmap_size=16)
    p0 = random_params(net, 21, table_scale=0.5, mlp_scale=0.15)
    n = 6000
    v = nb.synth(31, n)
    loss = run_step(net, v, n)
    g = net.get_grads()
    g64, l64 = O.train_grads(net.config, p0, v, v["target"], "f64")
    assert loss[0] == pytest.approx(l64[0], rel=1e-5)
    assert loss[1] == pytest.approx(l64[1], rel=1e-4, abs=1e-12)
    ntab, nst, nrr = net.param_layout()
    for name, sl in (("table", slice(0, ntab)), ("statnet", slice(ntab, ntab + nst)),
                     ("rrsnet", slice(ntab + nst, ntab + nst + nrr))):
        if name == "rrsnet" and step < 3:
            assert not np.any(g[sl]), name
            continue
        e = rel_err(g[sl].astype(np.float64), g64[sl])
        assert e < 2e-4, (name, e)
    # Adam (t = 1) applied to the GPU's own gradients
    p1 = net.get_params()
    pe = p0.copy()
    m = np.zeros_like(pe); vv = np.zeros_like(pe)
    count = ntab + nst + (nrr if step >= 3 else 0)
    O.adam(net.config, pe, g, m, vv, 1, 0, count)
    assert np.allclose(p1, pe, rtol=1e-5, atol=1e-7)
    if step < 3:
        assert np.array_equal(p1[ntab + nst:], p0[ntab + nst:])
    m1, v1, t = net.get_adam_state()
    assert t == 1
    assert np.allclose(m1[:count], 0.1 * g[:count], rtol=1e-5, atol=1e-12)
    net.close()


@pytest.mark.parametrize("shape", ["w64h3", "w128h3"])
def test_fp32_other_shapes_grads(shape):
    kw = {"w64h3": dict(statnet_width=64, statnet_hidden=3, rrsnet_width=64, rrsnet_hidden=3),
          "w128h3": dict(statnet_width=128, statnet_hidden=3, rrsnet_width=128, rrsnet_hidden=3)}[shape]
    net = make_net(max_train=1 << 13, log2_hashmap_size=15, **kw)
    p0 = random_params(net, 22, table_scale=0.5, mlp_scale=0.1)
    n = 3000
    v = nb.synth(32, n)
    loss = run_step(net, v, n)
    g = net.get_grads()
    g64, l64 = O.train_grads(net.config, p0, v, v["target"], "f64")
    assert loss == pytest.approx(l64, rel=1e-4)
    assert rel_err(g.astype(np.float64), g64) < 2e-4
    net.close()


def test_loss_decreases_over_steps():
    net = make_net(max_train=1 << 14)
    n = 8192
    v = nb.synth(33, n)
    losses = [run_step(net, v, n) for _ in range(30)]
    assert losses[-1][0] < 0.8 * losses[0][0], (losses[0], losses[-1])
    assert losses[-1][1] < losses[0][1], (losses[0], losses[-1])
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


def test_full_batch_262144_runs_and_is_finite():
    net = make_net(max_train=262144)
    v = nb.synth(34, 262144)
    loss = run_step(net, v, 262144)
    assert np.all(np.isfinite(loss)) and loss[0] > 0 and loss[1] > 0
    g = net.get_grads()
    assert np.all(np.isfinite(g))
    net.close()


MIXED_SHAPES = {
    # shape: (network kwargs, MLP init scale, error bars: table, StatNet, RRSNet)
    # measured on this batch: w64h2 2.3e-2 / 6.7e-3 / 4.1e-3, w64h3 3.0e-2 / 8.8e-3 / 3.6e-3,
    # w128h3 3.1e-2 / 8.3e-3 / 3.9e-3 (FP32 path: 4e-7)
    "w64h2": (dict(), 0.15, (4e-2, 1.5e-2, 1e-2)),
    "w64h3": (dict(statnet_width=64, statnet_hidden=3, rrsnet_width=64, rrsnet_hidden=3), 0.15,
              (5e-2, 1.5e-2, 1e-2)),
    "w128h3": (dict(statnet_width=128, statnet_hidden=3, rrsnet_width=128, rrsnet_hidden=3), 0.1,
               (5e-2, 1.5e-2, 1e-2)),
}


@pytest.mark.parametrize("shape", list(MIXED_SHAPES))
@pytest.mark.parametrize("prec", [nb.PREC_FP16, nb.PREC_BF16], ids=["fp16", "bf16"])
@pytest.mark.parametrize("step", [3, 2])
def test_mixed_training_vs_fp64_oracle(prec, step, shape):
    """tensor-core training step: FP16 StatNet / BF16 RRSNet MMAs with FP32 accumulation.
    Stated error bars (relative L2 norm of the gradient error, per parameter group)."""
    kw, mlp_scale, (bt, bs, br) = MIXED_SHAPES[shape]
    net = make_net(precision=prec, max_train=1 << 14, step=step, log2_hashmap_size=16, **kw)
    p0 = random_params(net, 21, table_scale=0.5, mlp_scale=mlp_scale)
    n = 6000
    v = nb.synth(31, n)
    loss = run_step(net, v, n)
    g = net.get_grads()
    g64, l64 = O.train_grads(net.config, p0, v, v["target"], "f64")
    assert loss[0] == pytest.approx(l64[0], rel=1e-4)
    assert loss[1] == pytest.approx(l64[1], rel=1e-3, abs=1e-12)
    ntab, nst, nrr = net.param_layout()
    bars = {"table": bt, "statnet": bs, "rrsnet": br}
    for name, sl in (("table", slice(0, ntab)), ("statnet", slice(ntab, ntab + nst)),
                     ("rrsnet", slice(ntab + nst, ntab + nst + nrr))):
        if name == "rrsnet" and step < 3:
            assert not np.any(g[sl])
            continue
        e = rel_err(g[sl].astype(np.float64), g64[sl])
        assert e < bars[name], (name, e)
    # Adam (t = 1) on the step's own gradients: the table part runs level group by level group
    # on the side stream, the MLP part after the join
    p1 = net.get_params()
    pe = p0.copy()
    m = np.zeros_like(pe); vv = np.zeros_like(pe)
    count = ntab + nst + (nrr if step >= 3 else 0)
    O.adam(net.config, pe, g, m, vv, 1, 0, count)
    assert np.allclose(p1, pe, rtol=1e-5, atol=1e-7)
    m1, _, t = net.get_adam_state()
    assert t == 1 and np.allclose(m1[:count], 0.1 * g[:count], rtol=1e-5, atol=1e-12)
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


def test_mixed_loss_decreases_and_matches_fp32_trajectory():
    torch = torch_cuda()
    nets = [make_net(max_train=1 << 14, precision=p) for p in (nb.PREC_FP32, nb.PREC_FP16)]
    n = 8192
    v = nb.synth(35, n)
    traj = [[run_step(net, v, n) for _ in range(20)] for net in nets]
    for t in traj:
        assert t[-1][0] < 0.9 * t[0][0]
    # after 20 Adam steps the two precisions stay close
    assert traj[1][-1][0] == pytest.approx(traj[0][-1][0], rel=5e-2)
    for net in nets:
        net.close()


@pytest.mark.parametrize("shape", ["w64h2", "w128h3"])
def test_split_training_equals_fused(shape):
    """the level-major encoding + StatNet kernel + level-major scatter gives the fused kernel's
    losses exactly and its gradients up to the order of the FP32 additions"""
    kw, mlp_scale, _ = MIXED_SHAPES[shape]
    net = make_net(precision=nb.PREC_FP16, max_train=1 << 14, step=3, log2_hashmap_size=16, **kw)
    p0 = random_params(net, 24, table_scale=0.5, mlp_scale=mlp_scale)
    n = 9000
    v = nb.synth(36, n)
    torch = torch_cuda()
    d = upload(v)
    out = {}
    for split in (1, 0):
        net.set_train_split(split)
        assert net.train_split() == split
        net.set_params(p0)
        loss = torch.zeros(2, dtype=torch.float64, device="cuda")
        net.trainGrads(soa(d), d["target"], n, loss, stream())
        torch.cuda.synchronize()
        out[split] = (loss.cpu().numpy(), net.get_grads().astype(np.float64))
    assert np.array_equal(out[0][0], out[1][0])
    ntab, nst, nrr = net.param_layout()
    for sl in (slice(0, ntab), slice(ntab, ntab + nst), slice(ntab + nst, ntab + nst + nrr)):
        e = rel_err(out[1][1][sl], out[0][1][sl])
        assert e < 1e-5, (shape, sl, e)
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


def _batch_dev(v, extra):
    torch = torch_cuda()
    d = upload(v)
    arrays = {k: d[k] for k in ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth",
                                "ref_mean", "target")}
    for k, a in extra.items():
        arrays[k] = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    return arrays


def _weighted_arrays(n, seed):
    rng = np.random.default_rng(seed)
    rt = rng.uniform(0.1, 3.0, n).astype(np.float32)
    rt[rng.random(n) < 0.25] = -1.0
    return {"rrs_target": rt, "error": rng.uniform(0.0, 4.0, n).astype(np.float32),
            "error_for_avg": rng.uniform(0.0, 6.0, n).astype(np.float32),
            "number_samples": rng.integers(0, 9, n).astype(np.float32)}, \
        rng.uniform(0.1, 1.0, n).astype(np.float32)


@pytest.mark.parametrize("prec", [nb.PREC_FP32, nb.PREC_FP16, nb.PREC_BF16],
                         ids=["fp32", "fp16", "bf16"])
def test_train_step_batch_weighted_losses_vs_fp64_oracle(prec):
    """nrrs_train_step_batch with every per-sample side array, the error sum and the shipped
    gammas: losses and gradients (before the update) against the FP64 oracle's weighted losses."""
    torch = torch_cuda()
    net = make_net(precision=prec, max_train=1 << 14, step=3, log2_hashmap_size=16)
    p0 = random_params(net, 41, table_scale=0.5, mlp_scale=0.15)
    n = 6000
    v = nb.synth(42, n)
    extra, sw = _weighted_arrays(n, 43)
    b = _batch_dev(v, extra)
    n_pix = 1500
    esum = 2.5 * n_pix
    d_esum = torch.tensor([esum], dtype=torch.float32, device="cuda")
    lp = nb.default_loss_params(gamma1=0.01, gamma2=0.05, gamma3=0.02, gamma4=0.01, clamp_on=1,
                                clamp_max=3.0, n_pixels=n_pix)
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainStepBatch(nb.train_batch(**b), n, torch.from_numpy(sw).cuda(), d_esum, lp, loss,
                       stream())
    torch.cuda.synchronize()
    g = net.get_grads().astype(np.float64)
    ov = dict(v)
    ov.update(extra)
    ov["sample_weight"] = sw
    w, keep = O.loss_weights(ov, gammas=(0.01, 0.05, 0.02, 0.01), clamp_on=1, clamp_max=3.0,
                             error_mean=esum / n_pix)
    g64, l64 = O.train_grads(net.config, p0, v, v["target"], "f64", weights=w)
    l = loss.cpu().numpy()
    fp32 = prec == nb.PREC_FP32
    assert l[0] == pytest.approx(l64[0], rel=1e-5 if fp32 else 1e-4)
    assert l[1] == pytest.approx(l64[1], rel=1e-4 if fp32 else 2e-3)
    ntab, nst, nrr = net.param_layout()
    bars = ({"table": 2e-4, "statnet": 2e-4, "rrsnet": 2e-4} if fp32 else
            {"table": 4e-2, "statnet": 1.5e-2, "rrsnet": 1.5e-2})
    for name, sl in (("table", slice(0, ntab)), ("statnet", slice(ntab, ntab + nst)),
                     ("rrsnet", slice(ntab + nst, ntab + nst + nrr))):
        e = rel_err(g[sl], g64[sl])
        assert e < bars[name], (name, e)
    rc, flags = net.device_status(stream())
    assert rc == nb.OK and flags == 0
    net.close()


@pytest.mark.parametrize("prec", [nb.PREC_FP32, nb.PREC_FP16], ids=["fp32", "fp16"])
def test_train_step_batch_defaults_equal_train_step(prec):
    """with no side arrays and the default loss parameters the batch step is nrrs_train_step,
    and so is everything after it: the factors inferred with the updated weights (the weight
    images are rebuilt after the step) and the losses of a second step"""
    torch = torch_cuda()
    n = 5000
    v = nb.synth(44, n)
    dp = nb.default_decide()
    out = []
    for batch_form in (False, True):
        net = make_net(precision=prec, max_train=1 << 13, step=3, log2_hashmap_size=15)
        random_params(net, 45, table_scale=0.5, mlp_scale=0.15)
        b = _batch_dev(v, {})
        losses = []
        for _ in range(2):
            loss = torch.zeros(2, dtype=torch.float64, device="cuda")
            if batch_form:
                net.trainStepBatch(nb.train_batch(**b), n, None, None,
                                   nb.default_loss_params(), loss, stream())
            else:
                net.train(soa(b), b["target"], n, loss, stream())
            losses.append(loss)
            if len(losses) == 1:
                st, rr = empty(3 * n), empty(n)
                net.inference(soa(b), n, dp, st, rr, stream())
        torch.cuda.synchronize()
        out.append((np.stack([l.cpu().numpy() for l in losses]),
                    net.get_grads().astype(np.float64), net.get_params(), host(rr)[:n].copy()))
        net.close()
    (la, ga, pa, ra), (lb, gb, pb, rb) = out
    assert np.allclose(la, lb, rtol=1e-6, atol=0)
    assert rel_err(gb, ga) < 1e-6
    assert np.allclose(pa, pb, rtol=1e-5, atol=1e-7)
    assert np.allclose(ra, rb, rtol=1e-5, atol=1e-7)
