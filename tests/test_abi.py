"""CPU tests of the C-ABI library: it loads, exports every function include/nrrs.h declares,
refuses to run without an sm_100 device (no CPU fallback), and its host-side helpers behave."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import nrrs_b200 as nb


def test_exports_every_header_symbol():
    L = nb.lib()
    names = nb.header_functions()
    assert len(names) >= 24
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_config_defaults_match_workload():
    c = nb.default_config()
    assert (c.n_levels, c.n_features_per_level, c.log2_hashmap_size, c.base_resolution) == (16, 2, 19, 16)
    assert c.per_level_scale == pytest.approx(1.5)
    assert (c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden) == (64, 2, 64, 2)
    assert (c.lr, c.beta1, c.beta2) == pytest.approx((1e-2, 0.9, 0.99))
    assert c.eps == pytest.approx(1e-15)
    d = nb.default_decide()
    assert (d.clamp_min, d.clamp_max, d.use_ceil, d.scale_up) == pytest.approx((0.05, 8.0, 1, 0))


def test_status_strings():
    L = nb.lib()
    for code in range(-8, 1):
        assert L.nrrs_status_string(code)


def test_no_cpu_fallback(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(nb.NRRSError) as e:
        nb.NRRSNetwork(nb.default_config(max_queue=1024, max_train=1024))
    assert e.value.code == nb.ERR_NO_DEVICE


def test_create_rejects_bad_config():
    L = nb.lib()
    h = C.c_void_p()
    for kw in (dict(n_levels=8), dict(statnet_width=48), dict(precision=7), dict(max_queue=0),
               dict(sh_degree=3)):
        c = nb.default_config(**kw)
        rc = L.nrrs_create(C.byref(c), C.byref(h))
        assert rc in (nb.ERR_INVALID_ARG, nb.ERR_UNSUPPORTED), kw
        assert L.nrrs_last_error(None)


def test_synth_is_deterministic_and_range_consistent():
    a = nb.synth(0, 70000)
    b = nb.synth(0, 70000)
    c = nb.synth(0, 1000, first=65000)  # straddles a generator block
    for k in a:
        assert np.array_equal(a[k], b[k])
        assert np.array_equal(a[k][65000:66000], c[k])
    assert np.allclose(np.linalg.norm(a["wi"], axis=1), 1, atol=1e-6)
    assert 0 <= a["pos"].min() and a["pos"].max() < 1
    assert set(np.unique(a["depth"])) <= set(range(6))
    assert abs(np.log(a["thp"]).mean() + 1) < 0.02 and abs(np.log(a["thp"]).std() - 1) < 0.02
    ff = (a["target"] > 0).all()
    assert ff


def test_header_declares_status_and_structs():
    text = nb.HEADER.read_text()
    for name in ("nrrs_config", "nrrs_vertex_soa", "nrrs_decide_params", "nrrs_segment"):
        assert f"}} {name};" in text
    assert C.sizeof(nb.Segment) == 24
    assert C.sizeof(nb.VertexSoA) == 9 * 8
    assert C.sizeof(nb.DecideParams) == 32
