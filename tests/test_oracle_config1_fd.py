"""Central finite differences (h = 1e-3, FP64) of the oracle's losses on 512 random parameters at
the full size of the training configuration: 262,144 samples, a 2^19-entry table, 64 wide x 2
hidden layers. The GPU paths are checked against these oracle gradients at the same size in
test_gpu_configs.py.

The StatNet loss is a mean of per-sample terms, and a table entry reaches only the samples with
a cell corner on its row. For the 448 table parameters the difference is therefore evaluated on
those samples alone and scaled by their share of the batch; the rows each sample touches are
recomputed here in numpy (the grid definition of the oracle: FP32 scaled coordinate, floor
clamped to [0, N-1], dense or spatial-hash index). The 32 StatNet and 32 RRSNet weights move
every sample and are differenced on the whole batch."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O

N = 262_144
H = 1e-3


def _corner_rows(cfg, pos):
    """[levels][n][8] table rows of every sample's cell corners."""
    lv, _ = O.level_table(cfg)
    p = np.clip(pos.astype(np.float32), np.float32(0), np.float32(1))
    mask = np.uint32((1 << cfg.log2_hashmap_size) - 1)
    out = []
    for offset, _, res, dense in lv:
        s = p * np.float32(res)
        c = np.clip(np.floor(s).astype(np.int64), 0, int(res) - 1).astype(np.uint32)
        rows = np.empty((p.shape[0], 8), np.uint32)
        for k in range(8):
            x = c[:, 0] + np.uint32(k & 1)
            y = c[:, 1] + np.uint32((k >> 1) & 1)
            z = c[:, 2] + np.uint32((k >> 2) & 1)
            if dense:
                R = np.uint32(res + 1)
                idx = x + R * y + R * R * z
            else:
                idx = (x ^ (y * np.uint32(2654435761)) ^ (z * np.uint32(805459861))) & mask
            rows[:, k] = np.uint32(offset) + idx
        out.append(rows)
    return lv, out


def _sub(v, idx):
    return {k: np.ascontiguousarray(a[idx]) for k, a in v.items()}


def test_fd_512_parameters_at_training_size():
    cfg = O.default_config(max_train=N, log2_hashmap_size=19)
    npar, ntab, nst, nrr = O.param_count(cfg)
    rng = np.random.default_rng(64)
    p = np.empty(npar, np.float32)
    p[:ntab] = rng.uniform(-0.5, 0.5, ntab)
    p[ntab:] = rng.uniform(-0.15, 0.15, nst + nrr)
    v = O.synth(65, N)
    tgt = v["target"]
    O.set_threads(0)
    g, loss = O.train_grads(cfg, p, v, tgt, "f64")
    p64 = p.astype(np.float64)
    lv, rows = _corner_rows(cfg, v["pos"])
    # 28 touched table parameters per level, 32 StatNet and 32 RRSNet weights
    picks = []
    for l, (offset, entries, _, _) in enumerate(lv):
        lo, hi = 2 * int(offset), 2 * (int(offset) + int(entries))
        touched = lo + np.nonzero(g[lo:hi])[0]
        picks += list(rng.choice(touched, 28, replace=False))
    picks += list(ntab + rng.choice(nst, 32, replace=False))
    picks += list(ntab + nst + rng.choice(nrr, 32, replace=False))
    assert len(picks) == 512
    order = [np.argsort(r.ravel(), kind="stable") for r in rows]
    flat = [r.ravel()[o] for r, o in zip(rows, order)]

    def fd(k, which, h):
        if k < ntab:
            row = k // 2
            l = int(np.searchsorted(lv[:, 0].astype(np.int64), row, side="right") - 1)
            a = np.searchsorted(flat[l], row, side="left")
            b = np.searchsorted(flat[l], row, side="right")
            samples = np.unique(order[l][a:b] // 8)
            sv = _sub(v, samples)
            scale = samples.size / N
            l0 = O.train_loss(cfg, p64, sv, sv["target"])[which]
        else:
            sv, scale, l0 = v, 1.0, full0[which]
        q = p64.copy()
        q[k] += h
        lp = O.train_loss(cfg, q, sv, sv["target"])[which]
        q[k] -= 2 * h
        lm = O.train_loss(cfg, q, sv, sv["target"])[which]
        return scale * (lp - lm) / (2 * h), scale * lp, scale * lm, scale * l0

    full0 = O.train_loss(cfg, p64, v, tgt)

    bad = []
    for k in picks:
        which = 1 if k >= ntab + nst else 0     # RRSNet weights -> RRS loss, else StatNet loss
        f, lp, lm, l0 = fd(k, which, H)
        floor = 1e-11 * max(1.0, loss[which]) / H
        kinked = abs((lp - l0) - (l0 - lm)) > 1e-3 * (abs(lp - l0) + abs(l0 - lm)) + H * floor
        ok = abs(f - g[k]) <= 1e-3 * max(abs(f), abs(g[k])) + floor
        if kinked or not ok:
            # a stencil across a ReLU kink or a cell boundary, or a strongly curved loss: again
            # with a stencil small enough to stay on one side
            hs = 1e-6
            f, *_ = fd(k, which, hs)
            floor = 1e-11 * max(1.0, loss[which]) / hs
            ok = abs(f - g[k]) <= 1e-4 * max(abs(f), abs(g[k])) + floor
        if not ok:
            bad.append((int(k), f, float(g[k])))
    assert not bad, bad[:10]
