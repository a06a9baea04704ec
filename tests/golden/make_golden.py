"""Generate tests/golden/*.json: hand-derived known-answer vectors for the NRRS decision path.

The reference (banbao990/NRRS-Code) ships no tests, no fixtures and cannot be built here
(OptiX, KiRaRay and tiny-cuda-nn are absent), so these vectors are derived directly from the
reference formulas, written out below in float32 numpy arithmetic independent of the C oracle:

  activationSigma        src/render/nrrs/net/networkcommon.h:61-68
  box_cox_transform      src/render/nrrs/train.cu:19-39 (lambda 0.5)
  RRSWeightWindow        src/render/common/commoncudautils.h:14-28
  normalizeSpatialCoord  src/render/nrc/nrctrain.h:111-115
  decision / emission    src/render/nrrs/integrator.cpp:1368-1460, commonworkqueue.h:19-25

Each decision case also lists the expected split counts worked out by hand in its comment.
Run: python tests/golden/make_golden.py  (rewrites the JSON files next to this script).
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

F = np.float32
HERE = Path(__file__).resolve().parent


def act_sigma(x):
    x = F(x)
    # FP32 op sequence of the reference: logf(1.0f + expf(x)) for x < 0
    if x < 0:
        return F(math.log(float(F(F(1.0) + F(math.exp(float(x)))))))
    return F(F(0.5) * x + F(0.6931471805599453))


def box_cox(x):
    return F(F(2.0) * (F(math.sqrt(float(F(x)))) - F(1.0)))


def weight_window(x, ww=5.0):
    x, ww = F(x), F(ww)
    dminus = F(F(2) / (F(1) + ww))
    dplus = F(dminus * ww)
    if x < dminus:
        return F(x / dminus)
    if x > dplus:
        return F(x / dplus)
    return F(1.0)


def normalize_pos(p, lo, hi):
    lo = np.array(lo, F)
    hi = np.array(hi, F)
    dg = (hi - lo).astype(F)
    infl = F(F(math.sqrt(float(F(F(dg[0] * dg[0] + dg[1] * dg[1]) + dg[2] * dg[2])))) * F(0.005))
    lo2, hi2 = (lo - infl).astype(F), (hi + infl).astype(F)
    c = ((lo2 + hi2) * F(0.5)).astype(F)
    d = (hi2 - lo2).astype(F)
    out = (F(0.5) + (np.array(p, F) - c) / d).astype(F)
    return np.clip(out, 0, 1).astype(F)


def decide(rrs, rnd, budget, nspec, use_ceil, rate, scale_up, sidx=None, capacity=None):
    rrs = np.array(rrs, F)
    rnd = np.array(rnd, F)
    terms = np.ceil(rrs).astype(F) if use_ceil else rrs
    total_sum = float(np.sum(terms.astype(np.float64)))  # exact for these small cases
    rcp = F(F(1.0) / F(total_sum))
    bud = F((budget - nspec) % (1 << 32))
    nf = F(bud * rcp)
    nf = F(nf * (F(1.0) if use_ceil else F(rate)))
    scale = nf if scale_up else (nf if nf < F(1.0) else F(1.0))
    queue, split, norm = [], [], {}
    for i in range(rrs.size):
        r = F(rrs[i] * scale)
        stid = int(sidx[i]) if sidx is not None else i
        norm[stid] = float(r)
        s = int(r)
        frac = F(r - F(s))
        s += 1 if rnd[i] <= frac else 0
        split.append(s)
        queue += [stid] * s
    total = len(queue)
    flags = 0
    if capacity is not None and total > capacity:
        queue = queue[:capacity]
        flags |= 0x1
    return {"split": split, "queue": queue, "total": total, "rrs_norm": norm, "flags": flags}


def main():
    ka = {
        "activation_sigma": [[x, float(act_sigma(x))] for x in (-10.0, -1.0, -0.5, 0.0, 0.5, 1.0, 10.0)],
        # 2 (sqrt(x) - 1): exact for perfect squares
        "box_cox": [[x, float(box_cox(x))] for x in (0.0, 0.25, 1.0, 4.0, 100.0, 0.5)],
        # dminus = 1/3, dplus = 5/3: 0.1 -> 0.3, 1 -> 1, 3 -> 1.8
        "weight_window": [[x, 5.0, float(weight_window(x))] for x in (0.1, 0.3, 1.0, 1.6, 3.0, 10.0)],
        # AABB [0,2]x[0,4]x[0,4]: |diag| = 6, inflation 0.03, centre (1,2,2), size (2.06, 4.06, 4.06)
        "normalize_pos": [
            {"lo": [0, 0, 0], "hi": [2, 4, 4], "p": [1.5, 1.0, 3.0],
             "out": normalize_pos([1.5, 1.0, 3.0], [0, 0, 0], [2, 4, 4]).tolist()},
            {"lo": [-1, -1, -1], "hi": [1, 1, 1], "p": [-5.0, 0.0, 0.999],
             "out": normalize_pos([-5.0, 0.0, 0.999], [-1, -1, -1], [1, 1, 1]).tolist()},
        ],
    }
    cases = []

    def add(name, comment, expect_split=None, **kw):
        res = decide(**kw)
        if expect_split is not None:
            assert res["split"] == expect_split, (name, res["split"], expect_split)
        case = {"name": name, "comment": comment, **kw, **res}
        cases.append(case)

    # sum 4, nf = 4 * 0.25 * rate 1 = 1 -> scale 1; s = [1, 2, 1 (0.5 <= 0.5), 0]
    add("plain", "rnd <= frac uses <=; scale = min(nf,1) = 1",
        expect_split=[1, 2, 1, 0],
        rrs=[1.0, 2.0, 0.5, 0.5], rnd=[0.9, 0.1, 0.5, 0.50000006], budget=4, nspec=0,
        use_ceil=False, rate=1.0, scale_up=False)
    # ceil sum 1+2+2 = 5, bud = 6-2 = 4, nf = 0.8 -> r = [0.24, 0.96, 1.6]; s = [1, 0, 2]
    add("ceil_specular", "use_ceil: rate ignored; n_specular reduces the budget",
        expect_split=[1, 0, 2],
        rrs=[0.3, 1.2, 2.0], rnd=[0.2, 0.97, 0.6], budget=6, nspec=2, use_ceil=True, rate=0.85,
        scale_up=False)
    # sum 1, nf = 4 * 1 * 0.5 = 2 (scale_up) -> r = [1, 1]; s = [2 (0 <= 0), 1]
    add("scale_up", "donnot_normalize_when_less_than_one = false lets nf > 1",
        expect_split=[2, 1],
        rrs=[0.5, 0.5], rnd=[0.0, 0.3], budget=4, nspec=0, use_ceil=False, rate=0.5,
        scale_up=True)
    # nf = 2 but min(nf,1) = 1 -> r = [0.5, 0.5]; s = [1, 0]
    add("no_scale_up", "nf > 1 is capped at 1 by default",
        expect_split=[1, 0],
        rrs=[0.5, 0.5], rnd=[0.0, 0.75], budget=4, nspec=0, use_ceil=False, rate=0.5,
        scale_up=False)
    # ceil sum 3, nf 1 -> r = 1, s = 1 each; queue carries the scatter indices
    add("scatter_index", "queue holds mScatterQueueIndex values; rrs_norm indexed by it",
        expect_split=[1, 1, 1],
        rrs=[1.0, 1.0, 1.0], rnd=[0.5, 0.5, 0.5], budget=3, nspec=0, use_ceil=True, rate=0.85,
        scale_up=False, sidx=[7, 3, 5])
    add("overflow", "capacity 3 < 4 copies: 3 written, total reports 4, overflow flag",
        expect_split=[1, 2, 1, 0],
        rrs=[1.0, 2.0, 0.5, 0.5], rnd=[0.9, 0.1, 0.5, 0.50000006], budget=4, nspec=0,
        use_ceil=False, rate=1.0, scale_up=False, capacity=3)
    # budget 2 - n_specular 3 wraps as uint32 like the reference: nf huge, min(nf,1) = 1
    add("specular_wrap", "uint32 budget - n_specular wraps as in integrator.cpp:1376",
        expect_split=[1, 0],
        rrs=[0.5, 0.5], rnd=[0.25, 0.75], budget=2, nspec=3, use_ceil=False, rate=0.85,
        scale_up=False)
    # split cap 8 with normalisation below one: r = 8 * 0.5 = 4 exactly -> s = 4 + (rnd <= 0)
    add("split_cap", "clamped factor 8 halved by nf = 0.5",
        expect_split=[4, 5],
        rrs=[8.0, 8.0], rnd=[0.5, 0.0], budget=8, nspec=0, use_ceil=True, rate=0.85,
        scale_up=False)
    add("empty", "n = 0", expect_split=[],
        rrs=[], rnd=[], budget=10, nspec=0, use_ceil=True, rate=0.85, scale_up=False)

    (HERE / "known_answers.json").write_text(json.dumps(ka, indent=1) + "\n")
    (HERE / "decide_cases.json").write_text(json.dumps(cases, indent=1) + "\n")
    print("wrote", HERE / "known_answers.json", HERE / "decide_cases.json")


if __name__ == "__main__":
    main()
