"""The cell image of the dense hash-grid levels (nrrs_set_cell_image): every gather of a dense
level reads one 32-byte block holding the cell's 8 FP16 corner entries instead of four table
rows. The corner values and their summation order are the table's, so inference in each mode
and launch shape and the decision must be bit-identical with the image on and off, and so must
the training step's forward; the image must follow every update of the table."""
from __future__ import annotations

import numpy as np
import pytest

import nrrs_b200 as nb
from gpu_util import empty, make_net, random_params, soa, stream, torch_cuda, upload

pytestmark = pytest.mark.gpu

SHAPES = {
    # 16 levels, 2^19: levels 0..3 dense
    "64x2_fp16_t19": (nb.PREC_FP16, dict(log2_hashmap_size=19)),
    # the 4K configuration: 128 x 3, BF16, 2^22 (levels 0..5 dense)
    "128x3_bf16_t22": (nb.PREC_BF16, dict(statnet_width=128, statnet_hidden=3, rrsnet_width=128,
                                          rrsnet_hidden=3, log2_hashmap_size=22)),
}


def _infer_all(net, d, n, dp):
    torch = torch_cuda()
    n_stats = 6 if net.config.network == nb.NET_REFERENCE else 3   # L and L^2, or log-stats
    o = dict(st=empty(n_stats * n), rrs=empty(n), norm=empty(n), split=empty(n, "uint8"),
             q=empty(9 * n, "int32"), sz=empty(1, "int32"))
    net.generateRRSNumber(soa(d), d["rnd"], n, n, 0, dp, o["st"], o["rrs"], o["norm"],
                          o["split"], o["q"], 9 * n, o["sz"], stream())
    torch.cuda.synchronize()
    return o


@pytest.mark.parametrize("shape", list(SHAPES))
def test_cell_image_inference_is_bit_identical(shape):
    torch = torch_cuda()
    prec, kw = SHAPES[shape]
    net = make_net(precision=prec, max_queue=1 << 18, **kw)
    assert net.cell_image()
    random_params(net, 91, table_scale=0.5, mlp_scale=0.1)
    n = 100_003
    v = nb.synth(92, n)
    d = upload(v)
    dp = nb.default_decide()
    tried = 0
    for mode in (0, 1, 2, 3):
        try:
            net.set_infer_split(mode)
        except nb.NRRSError:
            continue
        for w in (1, 2):
            try:
                net.set_launch_shape(0, w)
            except nb.NRRSError:
                continue
            net.set_cell_image(False)
            ref = _infer_all(net, d, n, dp)
            net.set_cell_image(True)
            out = _infer_all(net, d, n, dp)
            tried += 1
            for k in ref:
                assert torch.equal(out[k], ref[k]), (shape, mode, w, k)
    assert tried >= 2
    assert net.device_status(stream()) == (nb.OK, 0)
    net.close()


@pytest.mark.parametrize("split", [True, False], ids=["split", "fused"])
def test_cell_image_training_and_rebuild_are_bit_identical(split):
    """the first training step's losses are bit-identical with the image on and off (its
    forward gathers the same values); after each of three steps the factors inferred with the
    image equal those inferred from the table rows on the same weights, so the image is rebuilt
    from the updated table after every Adam pass (the table gradient's atomic additions make
    the weights themselves differ run to run in the last bits)"""
    torch = torch_cuda()
    n = 20_000
    v = nb.synth(93, n)
    d = upload(v)
    dp = nb.default_decide()
    first = []
    for cells in (False, True):
        net = make_net(precision=nb.PREC_FP16, max_queue=1 << 16, max_train=1 << 15, step=3,
                       log2_hashmap_size=17)
        net.set_train_split(split)
        net.set_cell_image(cells)
        random_params(net, 94, table_scale=0.5, mlp_scale=0.15)
        for step in range(3):
            loss = torch.zeros(2, dtype=torch.float64, device="cuda")
            net.train(soa(d), d["target"], n, loss, stream())
            if step == 0:
                first.append(loss.cpu().numpy())
            if cells:
                with_image = _infer_all(net, d, n, dp)
                net.set_cell_image(False)
                from_rows = _infer_all(net, d, n, dp)
                net.set_cell_image(True)
                for k in with_image:
                    assert torch.equal(with_image[k], from_rows[k]), (step, k)
        assert net.device_status(stream()) == (nb.OK, 0)
        net.close()
    assert np.array_equal(first[0], first[1])


def test_reference_network_cell_image_is_bit_identical():
    """the shipped network (8 levels, scale 2.0, 2^19: levels 0..2 dense) on the tensor cores"""
    torch = torch_cuda()
    net = nb.NRRSNetwork(nb.reference_config(precision=nb.PREC_FP16, max_queue=1 << 17,
                                             max_train=1 << 14))
    rng = np.random.default_rng(95)
    ntab, nst, nrr = net.param_layout()
    net.set_params(np.concatenate([rng.uniform(-0.5, 0.5, ntab),
                                   rng.uniform(-0.2, 0.2, nst + nrr)]).astype(np.float32))
    n = 50_001
    v = nb.synth(96, n)
    d = upload(v)
    dp = nb.default_decide()
    net.set_cell_image(False)
    ref = _infer_all(net, d, n, dp)
    net.set_cell_image(True)
    out = _infer_all(net, d, n, dp)
    for k in ref:
        assert torch.equal(out[k], ref[k]), k
    net.close()


def test_fp32_context_has_no_cell_image():
    net = make_net(precision=nb.PREC_FP32, max_queue=1 << 12, max_train=1 << 12,
                   log2_hashmap_size=15)
    assert not net.cell_image()
    with pytest.raises(nb.NRRSError):
        net.set_cell_image(True)
    net.set_cell_image(False)
    net.close()
