"""Generate tests/golden/*.json: hand-derived known-answer vectors for the NRRS decision path.

The reference (banbao990/NRRS-Code) ships no tests, no fixtures and cannot be built here
(OptiX, KiRaRay and tiny-cuda-nn are absent), so these vectors are derived directly from the
reference formulas, written out below in float32 numpy arithmetic independent of the C oracle:

  activationSigma        src/render/nrrs/net/networkcommon.h:61-68
  box_cox_transform      src/render/nrrs/train.cu:19-39 (lambda 0.5)
  RRSWeightWindow        src/render/common/commoncudautils.h:14-28
  normalizeSpatialCoord  src/render/nrc/nrctrain.h:111-115
  decision / emission    src/render/nrrs/integrator.cpp:1368-1460, commonworkqueue.h:19-25
  path records, training data and sample weights
                         src/render/nrrs/workqueue.h:122-170, train.cu:432-592
  per-pixel error (weighted L, relative error, clamp, sqrt(spp), error sum)
                         src/render/nrrs/train.cu:344-430, integrator.cpp:2358-2471

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


def records_expected(case):
    """Sequential restatement of recordNode / recordRadiance / nrrs_generate_training_data /
    nrrs_calculate_sample_weight in Python with exact rational radiance sums, under the library's
    ordering rules (nodes and samples in input order; the lowest-index child keeps its target)."""
    from fractions import Fraction
    cap = case["capacity"]
    nodes = []          # dicts per node
    size, dropped = 0, 0
    node_outs = []
    for b in case["bounces"]:
        outs = []
        for i in range(len(b["pixel"])):
            p = b["parent"][i]
            if b["record"][i]:
                if size < cap:
                    nodes.append(dict(pos=b["pos"][i], wi=b["wi"][i], thp=b["thp"][i],
                                      rough=b["roughness"][i], parent=p, pixel=b["pixel"][i],
                                      rrs=b["rrs"][i], depth=b["depth"][i],
                                      rad=[Fraction(0)] * 3, bad=False))
                    outs.append(size)
                    size += 1
                else:
                    dropped += 1
                    outs.append(p)
            else:
                outs.append(p)
        node_outs.append(outs)
        for nd, c in zip(b["contrib_node"], b["contrib"]):
            if nd < 0 or nd >= size:
                continue
            finite = all(math.isfinite(x) for x in c)
            cur = nd
            while cur != -1:        # the chain walk of workqueue.h:127-134
                if finite:
                    nodes[cur]["rad"] = [r + Fraction(x) for r, x in zip(nodes[cur]["rad"], c)]
                else:
                    nodes[cur]["bad"] = True
                cur = nodes[cur]["parent"]
    first_child = {}
    for i, n in enumerate(nodes):
        if n["parent"] >= 0 and n["parent"] not in first_child:
            first_child[n["parent"]] = i
    prm = case["params"]
    img = case["image"]
    counts = [0] * len(img)
    batch = []
    for i, n in enumerate(nodes):
        L = []
        for ch in range(3):
            rad = F(float(n["rad"][ch]))
            th = F(n["thp"][ch])
            l = F(rad / th) if th > F(prm["thp_eps"]) else F(0)
            L.append(F(0) if l < 0 else l)
        mean = F(F(F(L[0] + L[1]) + L[2]) / F(3))
        same = bool(prm["dedupe_rrs_target"]) and n["parent"] >= 0 and first_child[n["parent"]] != i
        if n["bad"] or (prm["ignore_zero_l"] and not mean > 0):
            continue
        thp = [F(F(t) * F(n["rrs"])) if prm["copy_rrs_node"] else F(t) for t in n["thp"]]
        q = img[n["pixel"]]
        batch.append(dict(node=i, target=[float(x) for x in L], thp=[float(x) for x in thp],
                          rrs_target=-1.0 if same else float(F(n["rrs"])), pixel=n["pixel"],
                          ref_mean=float(F(F(F(F(q[0]) + F(q[1])) + F(q[2])) / F(3)))))
        if not same:
            counts[n["pixel"]] += 1
    weights = [float(F(F(1) / F(counts[b["pixel"]]))) if counts[b["pixel"]] else 0.0 for b in batch]
    return dict(size=size, dropped=dropped, node_outs=node_outs, batch=batch, counts=counts,
                weights=weights)


def records_cases():
    """Hand-built path trees. Worked answer of "tree" (dyadic values, all sums exact):
      bounce 0: v0 (px 0) and v2 (px 2) record nodes 0 and 1; v1 records nothing (node -1)
      bounce 1: two children of node 0 -> nodes 2, 3; one of node 1 -> node 4; v1's -> node 5
      radiance: node 2 (1, .5, .25), node 3 (.25, 0, 0), node 4 (2, 0, 0), node 5 NaN,
                node 0 = own (.5, .25, 0) + nodes 2, 3 = (1.75, .75, .25), node 1 = (2, 0, 0);
                v1's (1, 1, 1) is dropped (no node)
      L = rad / thp: node 0 (3.5, 1.5, 0: thp 1e-6 <= eps), node 1 (2, 0, 0), node 2 (4, 1, .5),
                node 3 (.5, 0, 0), node 4 (4, 0, 0); node 5 dropped (NaN)
      dedupe: node 3 is node 0's second child -> rrs target -1, not counted
      counts: px 0 -> nodes 0, 2 = 2; px 2 -> nodes 1, 4 = 2 -> every weight 1/2"""
    nan = float("nan")
    tree_bounces = [
        dict(pos=[[0.1, 0.2, 0.3], [0.4, 0.5, 0.6], [0.7, 0.8, 0.9]],
             wi=[[0.0, 0.0, 1.0], [0.0, 1.0, 0.0], [1.0, 0.0, 0.0]],
             roughness=[0.25, 0.5, 0.75], thp=[[0.5, 0.5, 1e-6], [1.0, 1.0, 1.0], [1.0, 1.0, 1.0]],
             depth=[0, 0, 0], pixel=[0, 1, 2], rrs=[2.0, 0.5, 0.5], record=[1, 0, 1],
             parent=[-1, -1, -1],
             contrib_node=[0, -1], contrib=[[0.5, 0.25, 0.0], [1.0, 1.0, 1.0]]),
        dict(pos=[[0.15, 0.25, 0.35], [0.45, 0.55, 0.65], [0.75, 0.85, 0.95], [0.05, 0.05, 0.05]],
             wi=[[0.6, 0.0, 0.8], [0.0, 0.6, 0.8], [0.8, 0.6, 0.0], [0.0, 0.0, -1.0]],
             roughness=[0.1, 0.2, 0.3, 0.4],
             thp=[[0.25, 0.5, 0.5], [0.5, 0.5, 0.5], [0.5, 1.0, 1.0], [1.0, 1.0, 1.0]],
             depth=[1, 1, 1, 1], pixel=[0, 0, 2, 1], rrs=[1.5, 1.5, 1.0, 0.75],
             record=[1, 1, 1, 1], parent=[0, 0, 1, -1],
             contrib_node=[2, 3, 4, 5],
             contrib=[[1.0, 0.5, 0.25], [0.25, 0.0, 0.0], [2.0, 0.0, 0.0], [nan, 0.0, 0.0]]),
    ]
    image = [[0.3, 0.6, 0.9, 1.0], [0.0, 0.0, 0.0, 1.0], [1.0, 2.0, 4.0, 1.0]]
    cases = []
    for name, comment, cap, prm in (
        ("tree", "dedupe, zero-L filter, thp * rrs, thp <= eps, NaN chain, no-node contribution",
         16, dict(ignore_zero_l=1, copy_rrs_node=1, dedupe_rrs_target=1, thp_eps=1e-5)),
        ("tree_plain", "the reference defaults: no filter, no dedupe, thp as recorded",
         16, dict(ignore_zero_l=0, copy_rrs_node=0, dedupe_rrs_target=0, thp_eps=1e-5)),
        ("tree_full", "capacity 5: v1's child is refused (dropped 1, node_out = parent -1)",
         5, dict(ignore_zero_l=1, copy_rrs_node=1, dedupe_rrs_target=1, thp_eps=1e-5)),
    ):
        case = dict(name=name, comment=comment, capacity=cap, params=prm, bounces=tree_bounces,
                    image=image)
        case["expect"] = records_expected(case)
        cases.append(case)
    return cases


def pixel_error_expected(case):
    """Float32 restatement of weighted L (first frame, STEP#1.1), nrrs_update_weighted_L and
    nrrs_calculate_error, with patches added in pixel order and the error sum exact."""
    from fractions import Fraction
    w, h, sc = case["frame_width"], case["frame_height"], case["scale"]
    pw, ph = w // sc, h // sc
    pl = [[F(x) for x in px] for px in case["pixel_l"]]
    spp = F(case["spp"])
    cur, first, acc = [], [], []
    for ps in range(pw * ph):
        x0, y0 = (ps % pw) * sc, (ps // pw) * sc
        c, f = [F(0)] * 3, [F(0)] * 3
        for dy in range(sc):
            for dx in range(sc):
                px = (y0 + dy) * w + x0 + dx
                c = [F(c[k] + pl[px][k]) for k in range(3)]
                f = [F(f[k] + F(pl[px][k] / spp)) for k in range(3)]
        cur.append(c)
        first.append(f)
        acc.append(case["spp"] * sc * sc)
    b = F(case["blend"])
    keep = F(F(1) - b)
    wl = []
    for ps in range(pw * ph):
        n = F(acc[ps])
        wl.append([F(F(first[ps][k] * keep) + F(F(cur[ps][k] / n) * b)) for k in range(3)])
    err, err_avg = [], []
    for ps in range(pw * ph):
        q = []
        for k in range(3):
            r = F(case["ref"][ps][k])
            d = F(wl[ps][k] - r)
            q.append(F(F(d * d) / F(F(r * r) + F(0.01))))
        e = F(F(F(q[0] + q[1]) + q[2]) / F(3))
        if case["clamp"]:
            e = F(100) if math.isnan(e) else min(e, F(100))
        err.append(e)
        if case["multiply_samples"]:
            e = F(e * F(math.sqrt(float(F(case["spp_patch"][ps])))))
        err_avg.append(e)
    total = sum(Fraction(float(e)) for e in err_avg)
    return dict(current=[[float(x) for x in c] for c in cur], acc=acc,
                first=[[float(x) for x in f] for f in first],
                weighted=[[float(x) for x in v] for v in wl],
                error=[float(e) for e in err], error_for_avg=[float(e) for e in err_avg],
                sum=float(F(float(total))))


def pixel_error_cases():
    """Worked values of "patch2x2": frame 4x2, patches of 2x2 pixels, spp 2.
      patch 0 (pixels 0,1,4,5): pixel L (1,2,0.5) (3,0,0.5) (0,2,1) (4,4,0) -> current (8,8,2),
        acc 8, first frame sum of L/2 = (4,4,1); blend 0.5: 0.5*(4,4,1) + 0.5*(1,1,0.25)
        = (2.5, 2.5, 0.625)
      patch 1 (pixels 2,3,6,7): all L 0 -> current 0, weighted 0
      errors against ref (2.5,2.5,0.625) and (0,0,0): 0 and 0 (clamp on, no sample scaling)"""
    nan = float("nan")
    cases = [
        dict(name="patch2x2", frame_width=4, frame_height=2, scale=2, spp=2, blend=0.5,
             clamp=1, multiply_samples=0,
             pixel_l=[[1, 2, 0.5], [3, 0, 0.5], [0, 0, 0], [0, 0, 0],
                      [0, 2, 1], [4, 4, 0], [0, 0, 0], [0, 0, 0]],
             ref=[[2.5, 2.5, 0.625, 1], [0, 0, 0, 1]], spp_patch=[8, 8]),
        dict(name="clamp_nan_sqrt", frame_width=2, frame_height=2, scale=1, spp=1, blend=0.25,
             clamp=1, multiply_samples=1,
             # pixel 0: error 100*(2^2+...)/3 far above 100 -> clamped; pixel 1: NaN -> 100;
             # pixel 2: small error scaled by sqrt(9) = 3; pixel 3: exact match -> 0
             pixel_l=[[2, 2, 2], [nan, 0, 0], [1.5, 0.5, 1], [0.25, 0.5, 0.75]],
             ref=[[0, 0, 0, 1], [1, 1, 1, 1], [1, 1, 1, 1], [0.25, 0.5, 0.75, 1]],
             spp_patch=[4, 1, 9, 16]),
        dict(name="no_clamp", frame_width=2, frame_height=1, scale=1, spp=4, blend=0.5,
             clamp=0, multiply_samples=0,
             pixel_l=[[8, 8, 8], [4, 0, 0]], ref=[[0, 0, 0, 0], [1, 0, 0, 0]],
             spp_patch=[1, 1]),
    ]
    for c in cases:
        c["expect"] = pixel_error_expected(c)
    return cases


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
    pe = pixel_error_cases()
    (HERE / "pixel_error_cases.json").write_text(json.dumps(pe, indent=1, allow_nan=True) + "\n")
    rc = records_cases()
    (HERE / "records_cases.json").write_text(json.dumps(rc, indent=1, allow_nan=True) + "\n")
    (HERE / "decide_cases.json").write_text(json.dumps(cases, indent=1) + "\n")
    print("wrote", HERE / "known_answers.json", HERE / "decide_cases.json",
          HERE / "records_cases.json")


if __name__ == "__main__":
    main()
