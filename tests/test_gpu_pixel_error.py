"""GPU parity of the per-pixel error entry points (nrrs_count_patch_samples,
nrrs_accumulate_weighted_l, nrrs_update_weighted_l, nrrs_calculate_error) against the oracle, bit
for bit, and of the error gathers of nrrs_generate_training_data: the hand-derived cases, whole
frames of 1920x1080 (one-pixel patches) and 640x360 (2x2 and 4x4 patches) over two training
frames, the exact error sum on two calls in a row, and the batch's error, error_for_avg and
number_samples with the film read at each sample's patch."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import nrrs_b200 as nb
import oracle as O
from gpu_util import host, stream, torch_cuda
from test_gpu_records import GpuNodes, dev
from test_pixel_error_oracle import PE_CASES, params_of, same_f32

pytestmark = pytest.mark.gpu


class GpuError:
    """The device buffers of the per-pixel error of one frame size."""

    def __init__(self, p: nb.PixelErrorParams):
        torch = torch_cuda()
        self.p = p
        self.npix = p.frame_width * p.frame_height
        self.np = self.npix // max(p.scale, 1) ** 2
        self.wl = torch.zeros((self.np, 3), dtype=torch.float32, device="cuda")
        self.cur = torch.full((self.np, 3), -5.0, dtype=torch.float32, device="cuda")
        self.acc = torch.zeros(self.np, dtype=torch.int32, device="cuda")
        self.err = torch.full((2 * self.npix,), -5.0, dtype=torch.float32, device="cuda")
        self.spp = torch.zeros(self.np, dtype=torch.float32, device="cuda")
        self.sum = torch.zeros(C.sizeof(nb.ErrorSum), dtype=torch.uint8, device="cuda")

    def frame(self, pixel_l, spp: int, first: bool, ref, rays=None):
        s = stream()
        if rays is not None:
            self.spp.zero_()
            nb.count_patch_samples(self.p, dev(rays), len(rays), self.spp, s)
        nb.accumulate_weighted_l(self.p, dev(pixel_l), spp, first, self.wl, self.cur, self.acc, s)
        nb.update_weighted_l(self.p, self.cur, self.acc, self.wl, s)
        nb.calculate_error(self.p, dev(ref), ref.shape[1], self.wl, self.spp, self.err, self.sum,
                           s)
        raw = host(self.sum)
        value = raw[28:32].view(np.float32)[0]
        assert not raw[:28].any()            # the accumulators are left at zero
        return value


class HostError:
    def __init__(self, p: nb.PixelErrorParams):
        self.p = p
        self.npix = p.frame_width * p.frame_height
        self.np = self.npix // max(p.scale, 1) ** 2
        self.wl = np.zeros((self.np, 3), np.float32)
        self.cur = np.zeros((self.np, 3), np.float32)
        self.acc = np.zeros(self.np, np.uint32)
        self.err = np.zeros(2 * self.npix, np.float32)
        self.spp = np.zeros(self.np, np.float32)

    def frame(self, pixel_l, spp: int, first: bool, ref, rays=None):
        if rays is not None:
            self.spp[:] = 0
            O.count_patch_samples(self.p, rays, self.spp)
        O.accumulate_weighted_l(self.p, pixel_l, spp, first, self.wl, self.cur, self.acc)
        O.update_weighted_l(self.p, self.cur, self.acc, self.wl)
        return O.calculate_error(self.p, ref, self.wl, self.spp, self.err)


@pytest.mark.parametrize("case", PE_CASES, ids=[c["name"] for c in PE_CASES])
def test_gpu_pixel_error_golden(case):
    p = params_of(case)
    g = GpuError(p)
    g.spp.copy_(torch_cuda().tensor(case["spp_patch"], dtype=torch_cuda().float32))
    total = g.frame(np.array(case["pixel_l"], np.float32), case["spp"], True,
                    np.array(case["ref"], np.float32))
    e = case["expect"]
    assert same_f32(host(g.wl), e["weighted"])
    err = host(g.err)
    assert same_f32(err[:g.np], e["error"])
    assert same_f32(err[g.npix:g.npix + g.np], e["error_for_avg"])
    assert np.float32(total) == np.float32(e["sum"])


def synth_frame(rng, w, h, np_, spp):
    pixel_l = (rng.lognormal(-1, 1.5, size=(w * h, 3)) * spp).astype(np.float32)
    pixel_l[rng.uniform(size=w * h) < 0.05] = 0
    ref = rng.lognormal(-1, 1.2, size=(np_, 4)).astype(np.float32)
    ref[rng.uniform(size=np_) < 0.02, :3] = 0
    rays = rng.integers(0, w * h, size=3 * w * h).astype(np.uint32)
    return pixel_l, ref, rays


@pytest.mark.parametrize("w,h,scale,clamp,mult", [(1920, 1080, 1, 1, 0), (640, 360, 2, 1, 1),
                                                  (640, 360, 4, 0, 1)])
def test_gpu_pixel_error_matches_oracle(w, h, scale, clamp, mult):
    p = nb.PixelErrorParams(w, h, scale, 0.5, clamp, mult)
    g, o = GpuError(p), HostError(p)
    rng = np.random.default_rng(w + scale)
    for frame in range(2):                      # the first-frame initialisation, then a blend
        pixel_l, ref, rays = synth_frame(rng, w, h, g.np, 4)
        tg = g.frame(pixel_l, 4, frame == 0, ref, rays)
        to = o.frame(pixel_l, 4, frame == 0, ref, rays)
        assert host(g.spp).tobytes() == o.spp.tobytes()
        assert host(g.cur).tobytes() == o.cur.tobytes()
        assert host(g.acc).view(np.uint32).tobytes() == o.acc.tobytes()
        assert host(g.wl).tobytes() == o.wl.tobytes()
        err = host(g.err)
        assert err[:g.np].tobytes() == o.err[:g.np].tobytes()
        assert err[g.npix:g.npix + g.np].tobytes() == o.err[g.npix:g.npix + g.np].tobytes()
        assert np.float32(tg).tobytes() == np.float32(to).tobytes()


def test_gpu_error_sum_nan_and_reuse():
    p = nb.PixelErrorParams(64, 64, 1, 0.5, 0, 0)
    g, o = GpuError(p), HostError(p)
    rng = np.random.default_rng(3)
    pixel_l, ref, _ = synth_frame(rng, 64, 64, g.np, 1)
    pixel_l[17, 1] = np.inf                     # without the clamp the error is not finite
    tg = g.frame(pixel_l, 1, True, ref)
    to = o.frame(pixel_l, 1, True, ref)
    assert np.isnan(tg) and np.isnan(to)
    # the next call sums afresh: with a first-frame estimate (the blend would carry the Inf
    # on) every error is finite again, and the left-over accumulators must not leak in
    pixel_l[17, 1] = 0.5
    tg = g.frame(pixel_l, 1, True, ref)
    to = o.frame(pixel_l, 1, True, ref)
    assert np.float32(tg) == np.float32(to) and np.isfinite(tg)


@pytest.mark.parametrize("scale", [1, 2])
def test_gpu_batch_gathers_the_pixel_error(scale):
    """The batch's error, error_for_avg and number_samples and its ref_mean read at each
    sample's patch (train.cu:528-543), against the oracle."""
    torch = torch_cuda()
    W, H = 120, 80
    P = W * H
    bounces, _ = nb.synth_paths(101 + scale, P, capacity=4 * P)
    rng = np.random.default_rng(scale)
    npatch = P // scale ** 2
    image = rng.uniform(0, 2, size=(npatch, 4)).astype(np.float32)
    err = rng.uniform(0, 5, size=2 * P).astype(np.float32)
    spp = rng.integers(1, 30, size=npatch).astype(np.float32)
    dev_err, dev_spp = dev(err), dev(spp)
    prm_g = nb.default_train_data_params(copy_rrs_node=1, dedupe_rrs_target=1, frame_width=W,
                                         error_image_scale=scale,
                                         error_per_pixel=dev_err.data_ptr(),
                                         samples_per_patch=dev_spp.data_ptr())
    prm_o = nb.default_train_data_params(copy_rrs_node=1, dedupe_rrs_target=1, frame_width=W,
                                         error_image_scale=scale, error_per_pixel=err.ctypes.data,
                                         samples_per_patch=spp.ctypes.data)
    o = O.frame_training_data(bounces, image, 4 * P, prm_o, n_pixels=P)
    g = GpuNodes(4 * P, max(len(b["pixel"]) for b in bounces))
    for b in bounces:
        g.record(b)
        g.radiance(b["contrib_node"], b["contrib"])
    cap = 4 * P
    outs = {k: torch.full((cap,), -3.0, device="cuda") for k in ("error", "error_for_avg",
                                                                  "number_samples", "ref_mean")}
    size = torch.zeros(1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(P, dtype=torch.int32, device="cuda")
    g.pn.generate_training_data(prm_g, nb.train_batch(**outs), cap, size, image=dev(image),
                                image_channels=4, n_pixels=P, pixel_samples=counts,
                                stream=stream())
    m = int(host(size)[0])
    assert m == o["total"] > 1000
    for k in outs:
        assert host(outs[k])[:m].tobytes() == o["batch"][k].tobytes(), k
    assert g.pn.status(stream())[2] == 0


@pytest.mark.parametrize("w,h,scale", [(1920, 1080, 1), (640, 360, 2)])
def test_gpu_ubs_error_matches_oracle(w, h, scale):
    """nrrs_ubs_error (nrrs_UBS_calc_error) and its exact sum, two calls in a row."""
    torch = torch_cuda()
    p = nb.PixelErrorParams(w, h, scale, 0.5, 1, 0)
    npix, npatch = w * h, (w // scale) * (h // scale)
    rng = np.random.default_rng(w)
    esum = torch.zeros(C.sizeof(nb.ErrorSum), dtype=torch.uint8, device="cuda")
    err = torch.full((npix,), -5.0, device="cuda")
    for spp in (1, 4):
        pixel_l = (rng.lognormal(-1, 1.5, size=(npix, 3)) * spp).astype(np.float32)
        ref = rng.lognormal(-1, 1.2, size=(npatch, 4)).astype(np.float32)
        nb.ubs_error(p, dev(pixel_l), spp, dev(ref), 4, err, esum, stream())
        want = np.zeros(npix, np.float32)
        total = O.ubs_error(p, pixel_l, spp, ref, want)
        assert host(err).tobytes() == want.tobytes()
        raw = host(esum)
        assert not raw[:28].any()
        assert raw[28:32].view(np.float32)[0] == np.float32(total)
