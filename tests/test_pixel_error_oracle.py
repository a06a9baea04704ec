"""CPU tests of the per-pixel error oracle (oracle/records.c): pinned to the hand-derived cases of
tests/golden/pixel_error_cases.json (weighted L, its blend, the relative error with its clamp and
sqrt(spp) copy, the exact error sum), plus the patch sample counts."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
PE_CASES = json.loads((GOLD / "pixel_error_cases.json").read_text())


def params_of(case) -> nb.PixelErrorParams:
    return nb.PixelErrorParams(case["frame_width"], case["frame_height"], case["scale"],
                               case["blend"], case["clamp"], case["multiply_samples"])


def same_f32(got, want):
    """Bit-equal float32 arrays, except that a NaN matches any NaN (the GPU's arithmetic gives
    its own NaN bit pattern)."""
    got = np.asarray(got, np.float32).ravel()
    want = np.asarray(want, np.float32).ravel()
    gn, wn = np.isnan(got), np.isnan(want)
    return bool((gn == wn).all()) and got[~gn].tobytes() == want[~wn].tobytes()


@pytest.mark.parametrize("case", PE_CASES, ids=[c["name"] for c in PE_CASES])
def test_oracle_pixel_error_matches_golden(case):
    p = params_of(case)
    npix = case["frame_width"] * case["frame_height"]
    npatch = npix // case["scale"] ** 2
    wl = np.zeros((npatch, 3), np.float32)
    cur = np.zeros((npatch, 3), np.float32)
    acc = np.zeros(npatch, np.uint32)
    O.accumulate_weighted_l(p, np.array(case["pixel_l"], np.float32), case["spp"], True, wl, cur,
                            acc)
    e = case["expect"]
    assert same_f32(cur, e["current"]) and acc.tolist() == e["acc"]
    assert same_f32(wl, e["first"])
    O.update_weighted_l(p, cur, acc, wl)
    assert same_f32(wl, e["weighted"])
    err = np.full(2 * npix, -1, np.float32)
    total = O.calculate_error(p, np.array(case["ref"], np.float32), wl,
                              np.array(case["spp_patch"], np.float32), err)
    assert same_f32(err[:npatch], e["error"])
    assert same_f32(err[npix:npix + npatch], e["error_for_avg"])
    assert np.float32(total) == np.float32(e["sum"])


def test_oracle_patch_counts_and_nan_sum():
    p = nb.PixelErrorParams(6, 4, 2, 0.5, 0, 0)
    spp = np.zeros(6, np.float32)
    O.count_patch_samples(p, np.array([0, 1, 6, 7, 23, 23, 99], np.uint32), spp)
    # pixels 0, 1, 6, 7 are patch 0; 23 (x 5, y 3) is patch 5; 99 is outside the frame
    assert spp.tolist() == [4, 0, 0, 0, 0, 2]
    # an error that is not finite makes the sum NaN (without the clamp)
    wl = np.array([[np.inf, 0, 0]] + [[0, 0, 0]] * 5, np.float32)
    err = np.zeros(48, np.float32)
    total = O.calculate_error(p, np.zeros((6, 3), np.float32), wl, None, err)
    assert math.isnan(total) and math.isinf(err[0])
