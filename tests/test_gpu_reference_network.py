"""GPU parity of the reference's shipped network (nrrs_config_reference_network,
common/configs/nrrs/nrrs/2net-simple.json): HashGrid 8 levels x 2 features (base 16, scale 2.0)
+ OneBlob 4 bins on the lat-long direction + OneBlob 8 bins on the warped roughness, 32-wide
LeakyReLU MLPs with 3 hidden layers, a 6-output StatNet (L, L^2) and the reference's glue.
Inference, the decision on the GPU's factors and the training step against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import empty, host, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu


def ref_net(**kw):
    base = dict(max_queue=1 << 20, max_train=1 << 16)
    base.update(kw)
    return nb.NRRSNetwork(nb.reference_config(**base))


def ref_params(net, seed, table_scale=0.5, mlp_scale=0.3):
    rng = np.random.default_rng(seed)
    ntab, nst, nrr = net.param_layout()
    p = np.concatenate([rng.uniform(-table_scale, table_scale, ntab),
                        rng.uniform(-mlp_scale, mlp_scale, nst + nrr)]).astype(np.float32)
    net.set_params(p)
    return p


def test_reference_network_layout_matches_oracle():
    net = ref_net()
    cfg = net.config
    assert (cfg.network, cfg.n_levels, cfg.statnet_width, cfg.statnet_hidden) == (1, 8, 32, 3)
    assert tuple(net.param_layout()) == tuple(O.param_count(cfg)[1:])
    assert np.array_equal(net.level_table(), O.level_table(cfg)[0])
    net.close()


@pytest.mark.parametrize("source", [nb.FACTOR_RRSNET, nb.FACTOR_ADRRS], ids=["rrsnet", "adrrs"])
def test_fp32_inference_and_decision_vs_oracle(source):
    torch = torch_cuda()
    net = ref_net(precision=nb.PREC_FP32)
    p = ref_params(net, 81)
    n = 100_003
    v = nb.synth(82, n)
    d = upload(v)
    dp = nb.default_decide(factor_source=source)
    cap = 9 * n
    st, rr, norm = empty(6 * n), empty(n), empty(n)
    split, q, sz = empty(n, "uint8"), empty(cap, "int32"), empty(1, "int32")
    net.generateRRSNumber(soa(d), d["rnd"], n, n, 0, dp, st, rr, norm, split, q, cap, sz, stream())
    torch.cuda.synchronize()
    g_st = host(st)[:6 * n].reshape(n, 6)
    g_rr = host(rr)[:n].copy()
    o32 = O.infer(net.config, p, v, dp, "f32", want=("stats", "rrs"))
    o64 = O.infer(net.config, p, v, dp, "f64", want=("stats", "rrs"))
    assert np.allclose(g_st, o32["stats"], rtol=2e-4, atol=2e-5)
    assert np.max(np.abs(g_rr - o64["rrs"]) / o64["rrs"]) < 1e-4
    # the decision on the GPU's factors: bit-exact against the oracle
    od = O.decide_emit(g_rr, v["rnd"], n, 0, dp, capacity=cap, shift_n=net.config.max_queue)
    tot = int(host(sz, np.uint32)[0])
    assert tot == od["total"]
    assert np.array_equal(host(split)[:n], od["split"])
    assert np.array_equal(host(q, np.uint32)[:tot], od["queue"])
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


@pytest.mark.parametrize("step", [3, 2])
def test_fp32_training_vs_fp64_oracle(step):
    torch = torch_cuda()
    net = ref_net(precision=nb.PREC_FP32, max_train=1 << 14, step=step, log2_hashmap_size=16)
    p = ref_params(net, 83)
    n = 6000
    v = nb.synth(84, n)
    d = upload(v)
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainGrads(soa(d), d["target"], n, loss, stream())
    torch.cuda.synchronize()
    g = net.get_grads().astype(np.float64)
    g64, l64 = O.train_grads(net.config, p, v, v["target"], "f64")
    l = loss.cpu().numpy()
    assert l[0] == pytest.approx(l64[0], rel=1e-4)
    assert l[1] == pytest.approx(l64[1], rel=1e-4, abs=1e-12)
    ntab, nst, nrr = net.param_layout()
    for name, sl in (("table", slice(0, ntab)), ("statnet", slice(ntab, ntab + nst)),
                     ("rrsnet", slice(ntab + nst, ntab + nst + nrr))):
        if name == "rrsnet" and step < 3:
            assert not np.any(g[sl])
            continue
        e = np.linalg.norm(g[sl] - g64[sl]) / max(np.linalg.norm(g64[sl]), 1e-30)
        assert e < 5e-4, (name, e)
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


def test_fp32_training_reduces_the_losses():
    torch = torch_cuda()
    net = ref_net(precision=nb.PREC_FP32, max_train=1 << 14)
    n = 8192
    v = nb.synth(85, n)
    d = upload(v)
    losses = []
    for _ in range(40):
        loss = torch.zeros(2, dtype=torch.float64, device="cuda")
        net.train(soa(d), d["target"], n, loss, stream())
        losses.append(loss.cpu().numpy())
    assert losses[-1][0] < 0.7 * losses[0][0], (losses[0], losses[-1])
    assert losses[-1][1] < losses[0][1], (losses[0], losses[-1])
    net.close()


@pytest.mark.parametrize("prec", [nb.PREC_FP16, nb.PREC_BF16], ids=["fp16", "bf16"])
@pytest.mark.parametrize("wgs", [1, 2])
def test_mixed_inference_vs_fp64_oracle(prec, wgs):
    """tensor-core inference (tcgen05, M = 128 x N = 32 tiles, FP16 table): factors within the
    workload's 1e-2 of the FP64 oracle, L and L^2 within 2e-2 x max(1, |y|); the decision on the
    GPU's factors bit-exact"""
    torch = torch_cuda()
    net = ref_net(precision=prec)
    net.set_launch_shape(0, wgs)
    p = ref_params(net, 86, mlp_scale=0.2)
    n = 65_536
    v = nb.synth(87, n)
    d = upload(v)
    dp = nb.default_decide()
    cap = 9 * n
    st, rr, norm = empty(6 * n), empty(n), empty(n)
    split, q, sz = empty(n, "uint8"), empty(cap, "int32"), empty(1, "int32")
    net.generateRRSNumber(soa(d), d["rnd"], n, n, 0, dp, st, rr, norm, split, q, cap, sz, stream())
    torch.cuda.synchronize()
    g_st = host(st)[:6 * n].reshape(n, 6)
    g_rr = host(rr)[:n].copy()
    o64 = O.infer(net.config, p, v, dp, "f64", want=("stats", "rrs"))
    assert np.max(np.abs(g_rr - o64["rrs"]) / o64["rrs"]) < 1e-2
    err = np.abs(g_st - o64["stats"]) / np.maximum(1.0, np.abs(o64["stats"]))
    assert err.max() < 2e-2, err.max()
    od = O.decide_emit(g_rr, v["rnd"], n, 0, dp, capacity=cap, shift_n=net.config.max_queue)
    tot = int(host(sz, np.uint32)[0])
    assert tot == od["total"]
    assert np.array_equal(host(q, np.uint32)[:tot], od["queue"])
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


def test_mixed_context_trains_on_the_fp32_kernels():
    """a mixed-precision context of the reference network trains with the FP32 step (its
    tensor-core step covers the workload's shapes only) and then infers on the tensor cores"""
    torch = torch_cuda()
    net = ref_net(precision=nb.PREC_FP16, max_train=1 << 14, log2_hashmap_size=16)
    p = ref_params(net, 88)
    n = 4000
    v = nb.synth(89, n)
    d = upload(v)
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainGrads(soa(d), d["target"], n, loss, stream())
    torch.cuda.synchronize()
    g = net.get_grads().astype(np.float64)
    g64, l64 = O.train_grads(net.config, p, v, v["target"], "f64")
    assert loss.cpu().numpy() == pytest.approx(l64, rel=1e-4)
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 5e-4
    net.close()


def test_adam_step_uses_the_per_network_learning_rates():
    """the shipped settings train the encoding and StatNet with lr 5e-3 and RRSNet with 5e-4
    (2net-simple.json level0 / level1): one step of the GPU equals the oracle's Adam on the
    GPU's own gradients, and the first step moves each parameter by its network's lr"""
    torch = torch_cuda()
    net = ref_net(precision=nb.PREC_FP32, max_train=1 << 14, log2_hashmap_size=16)
    cfg = net.config
    assert cfg.lr == pytest.approx(5e-3) and cfg.lr_rrsnet == pytest.approx(5e-4)
    p0 = ref_params(net, 90)
    n = 5000
    v = nb.synth(91, n)
    d = upload(v)
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.train(soa(d), d["target"], n, loss, stream())
    torch.cuda.synchronize()
    g = net.get_grads()
    p1 = net.get_params()
    pe = p0.copy()
    m = np.zeros_like(pe)
    vv = np.zeros_like(pe)
    O.adam(cfg, pe, g, m, vv, 1)
    assert np.allclose(p1, pe, rtol=1e-5, atol=1e-7)
    ntab, nst, nrr = net.param_layout()
    moved = np.abs(p1 - p0)
    big = np.abs(g) > 1e-6     # away from the eps and l2 corners of the first step
    st = slice(ntab, ntab + nst)
    rr = slice(ntab + nst, ntab + nst + nrr)
    assert np.allclose(moved[st][big[st]], 5e-3, rtol=2e-2)
    assert np.allclose(moved[rr][big[rr]], 5e-4, rtol=2e-2)
    net.close()


def test_weighted_training_step_batch_vs_fp64_oracle():
    """nrrs_train_step_batch on the shipped network with every per-sample side array, the error
    sum and the shipped gammas: losses and gradients against the FP64 oracle's weighted losses
    (FP32 kernels, the reference network's relative L2 StatNet loss)"""
    torch = torch_cuda()
    net = ref_net(precision=nb.PREC_FP32, max_train=1 << 14, log2_hashmap_size=16)
    p0 = ref_params(net, 92)
    n = 6000
    v = nb.synth(93, n)
    rng = np.random.default_rng(94)
    rt = rng.uniform(0.1, 3.0, n).astype(np.float32)
    rt[rng.random(n) < 0.25] = -1.0
    extra = {"rrs_target": rt, "error": rng.uniform(0.0, 4.0, n).astype(np.float32),
             "error_for_avg": rng.uniform(0.0, 6.0, n).astype(np.float32),
             "number_samples": rng.integers(0, 9, n).astype(np.float32)}
    sw = rng.uniform(0.1, 1.0, n).astype(np.float32)
    d = upload(v)
    b = {k: d[k] for k in ("pos", "wi", "normal", "roughness", "albedo", "thp", "depth",
                           "ref_mean", "target")}
    for k, a in extra.items():
        b[k] = torch.from_numpy(a).cuda()
    n_pix = 1500
    esum = 2.5 * n_pix
    d_esum = torch.tensor([esum], dtype=torch.float32, device="cuda")
    lp = nb.default_loss_params(gamma1=0.01, gamma2=0.05, gamma3=0.0, gamma4=0.01, clamp_on=1,
                                clamp_max=10.0, n_pixels=n_pix)
    loss = torch.zeros(2, dtype=torch.float64, device="cuda")
    net.trainStepBatch(nb.train_batch(**b), n, torch.from_numpy(sw).cuda(), d_esum, lp, loss,
                       stream())
    torch.cuda.synchronize()
    g = net.get_grads().astype(np.float64)
    ov = dict(v)
    ov.update(extra)
    ov["sample_weight"] = sw
    w, _ = O.loss_weights(ov, gammas=(0.01, 0.05, 0.0, 0.01), clamp_on=1, clamp_max=10.0,
                          error_mean=esum / n_pix)
    g64, l64 = O.train_grads(net.config, p0, v, v["target"], "f64", weights=w)
    lo = loss.cpu().numpy()
    assert lo[0] == pytest.approx(l64[0], rel=1e-4)
    assert lo[1] == pytest.approx(l64[1], rel=1e-4)
    ntab, nst, nrr = net.param_layout()
    for name, sl in (("table", slice(0, ntab)), ("statnet", slice(ntab, ntab + nst)),
                     ("rrsnet", slice(ntab + nst, ntab + nst + nrr))):
        e = np.linalg.norm(g[sl] - g64[sl]) / max(np.linalg.norm(g64[sl]), 1e-30)
        assert e < 5e-4, (name, e)
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()
