"""Where the mixed-precision training step's hash-table gradient error comes from.

The tensor-core StatNet step evaluates the forward pass with FP16 operands (hash features from
the FP16 table, FP16 weight images, FP16 activation tiles; FP32 accumulation) and the backward
with FP16 deltas. Its table gradient is 2-3 % off FP64 in relative L2 (tests/test_gpu_train.py,
tests/test_gpu_configs.py). This test replays the StatNet backward in numpy on the oracle's
FP64 inputs, rounding one stage at a time to FP16, and measures the relative L2 error of the
per-sample hash-lane gradients (the table gradient is a fixed linear map of them):

  * rounding only the deltas, or only the lane gradients, costs a few 1e-4;
  * rounding the forward (inputs, weights or activations) costs 1-2 % each, about 2 % together,
    the GPU's figure: a ReLU unit whose pre-activation lies within rounding of zero switches
    off or on, and the gradient of a ReLU network changes discontinuously with its masks;
  * a forward whose products are formed from split FP16 pairs (x = x_hi + x_lo, W = W_hi +
    W_lo, three products) brings the error back to a few 1e-4.

So the error is that of evaluating the network in FP16, not of the backward kernels."""
from __future__ import annotations

import numpy as np

import oracle as O


def _f16(a):
    return a.astype(np.float16).astype(np.float64)


def _split(a):
    h = _f16(a)
    return h, _f16(a - h)


def _mm3(x, w):
    xh, xl = _split(x)
    wh, wl = _split(w)
    return xh @ wh.T + xl @ wh.T + xh @ wl.T


def test_mixed_table_gradient_error_comes_from_the_fp16_forward():
    cfg = O.default_config(log2_hashmap_size=16, max_train=1 << 14)
    npar, ntab, nst, nrr = O.param_count(cfg)
    rng = np.random.default_rng(21)
    p = np.empty(npar, np.float32)
    p[:ntab] = rng.uniform(-0.5, 0.5, ntab)
    p[ntab:] = rng.uniform(-0.15, 0.15, nst + nrr)
    n = 6000
    v = O.synth(31, n)
    x0 = O.infer(cfg, p, v, O.default_decide(), "f64", want=("x0",))["x0"]
    _, l64 = O.train_grads(cfg, p, v, v["target"], "f64")
    W = p[ntab:ntab + nst].astype(np.float64)
    W0, W1, W2 = W[:4096].reshape(64, 64), W[4096:8192].reshape(64, 64), W[8192:].reshape(3, 64)
    tgt = np.log(v["target"].astype(np.float64) + cfg.stat_eps)

    def backward(x, w0, w1, w2, act=lambda a: a, mm=lambda a, b: a @ b.T, rd=lambda a: a):
        z1 = mm(x, w0)
        h1 = act(np.maximum(z1, 0))
        z2 = mm(h1, w1)
        h2 = act(np.maximum(z2, 0))
        y = mm(h2, w2)
        dy = rd(2 * (y - tgt) / 3.0)
        dh2 = rd((dy @ (w2 if mm is not _mm3 else _f16(w2))) * (z2 > 0))
        dh1 = rd((dh2 @ (w1 if mm is not _mm3 else _f16(w1))) * (z1 > 0))
        dx = dh1 @ (w0 if mm is not _mm3 else _f16(w0))
        return dx[:, :32], y

    ref, y = backward(x0, W0, W1, W2)
    # the restated backward is the oracle's: same StatNet loss
    assert abs(np.mean((y - tgt) ** 2) - l64[0]) < 1e-9 * l64[0]

    def rel(d):
        return float(np.linalg.norm(d - ref) / np.linalg.norm(ref))

    deltas = rel(backward(x0, W0, W1, W2, rd=_f16)[0])
    inputs = rel(backward(_f16(x0), W0, W1, W2)[0])
    weights = rel(backward(x0, _f16(W0), _f16(W1), _f16(W2))[0])
    acts = rel(backward(x0, W0, W1, W2, act=_f16)[0])
    forward = rel(backward(_f16(x0), _f16(W0), _f16(W1), _f16(W2), act=_f16, rd=_f16)[0])
    split = rel(backward(x0, W0, W1, W2, mm=_mm3, rd=_f16)[0])
    assert deltas < 1e-3, deltas
    for name, e in (("inputs", inputs), ("weights", weights), ("activations", acts)):
        assert 3e-3 < e < 5e-2, (name, e)
    assert 1e-2 < forward < 5e-2, forward
    assert split < 1e-3, split


def test_fp32_table_gradient_error_at_training_size_is_one_mask_flip():
    """The plain FP32 path at the training size (262,144 samples, 2^19 table) replayed in
    numpy float32: one hidden unit of one sample flips its ReLU mask against FP64, and that
    sample carries almost all of the hash-lane gradient error (about 5.7e-4 relative L2, the
    GPU's 5.1e-4)."""
    cfg = O.default_config(max_train=262_144, log2_hashmap_size=19)
    npar, ntab, nst, nrr = O.param_count(cfg)
    rng = np.random.default_rng(61)   # the draws of tests/test_gpu_configs.py's parameters
    p = np.empty(npar, np.float32)
    p[:ntab] = rng.uniform(-0.5, 0.5, ntab)
    p[ntab:] = rng.uniform(-0.15, 0.15, nst + nrr)
    n = 262_144
    v = O.synth(62, n)
    x0 = O.infer(cfg, p, v, O.default_decide(), "f64", want=("x0",))["x0"]
    W = p[ntab:ntab + nst].astype(np.float64)
    W0, W1, W2 = W[:4096].reshape(64, 64), W[4096:8192].reshape(64, 64), W[8192:].reshape(3, 64)
    tgt = np.log(v["target"].astype(np.float64) + cfg.stat_eps)

    def run(dt):
        x, a0, a1, a2, t = (m.astype(dt) for m in (x0, W0, W1, W2, tgt))
        z1 = x @ a0.T
        h1 = np.maximum(z1, 0)
        z2 = h1 @ a1.T
        y = np.maximum(z2, 0) @ a2.T
        dh2 = ((2 * (y - t) / 3) @ a2) * (z2 > 0)
        dh1 = (dh2 @ a1) * (z1 > 0)
        return (dh1 @ a0)[:, :32].astype(np.float64), (z1 > 0), (z2 > 0)

    a, m1a, m2a = run(np.float64)
    b, m1b, m2b = run(np.float32)
    flips = int(np.sum(m1a != m1b) + np.sum(m2a != m2b))
    per = np.linalg.norm(b - a, axis=1)
    rel = float(np.linalg.norm(b - a) / np.linalg.norm(a))
    assert flips >= 1
    assert 2e-4 < rel < 2e-3, rel
    assert per.max() ** 2 / (per ** 2).sum() > 0.99
