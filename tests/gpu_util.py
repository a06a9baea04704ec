"""Helpers shared by the GPU tests: upload synthetic vertices, run the library, compare."""
from __future__ import annotations

import numpy as np

import nrrs_b200 as nb


def torch_cuda():
    import torch
    return torch


def upload(v: dict, keys=nb.VERTEX_FIELDS + ("rnd", "target")):
    torch = torch_cuda()
    out = {}
    for k in keys:
        if k in v and v[k] is not None:
            a = v[k]
            if a.dtype == np.uint32:
                out[k] = torch.from_numpy(a.view(np.int32)).cuda()
            else:
                out[k] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return out


def soa(d: dict, scatter_index=None) -> nb.VertexSoA:
    return nb.vertex_soa(d["pos"], d["wi"], d["normal"], d["roughness"], d["albedo"], d["thp"],
                         d.get("depth"), d.get("ref_mean"), scatter_index)


def stream():
    return torch_cuda().cuda.current_stream().cuda_stream


def empty(n, dtype="float32"):
    torch = torch_cuda()
    dt = {"float32": torch.float32, "uint8": torch.uint8, "int32": torch.int32,
          "float64": torch.float64}[dtype]
    return torch.zeros(max(int(n), 1), dtype=dt, device="cuda")


def host(t, np_dtype=None):
    torch = torch_cuda()
    torch.cuda.synchronize()
    a = t.cpu().numpy()
    if np_dtype is not None:
        a = a.view(np_dtype)
    return a


def make_net(**kw) -> nb.NRRSNetwork:
    base = dict(max_queue=1 << 21, max_train=1 << 16)
    base.update(kw)
    return nb.NRRSNetwork(nb.default_config(**base))


def random_params(net: nb.NRRSNetwork, seed=0, table_scale=0.5, mlp_scale=0.2):
    rng = np.random.default_rng(seed)
    ntab, nst, nrr = net.param_layout()
    p = np.empty(ntab + nst + nrr, np.float32)
    p[:ntab] = rng.uniform(-table_scale, table_scale, ntab)
    p[ntab:] = rng.uniform(-mlp_scale, mlp_scale, nst + nrr)
    net.set_params(p)
    return p
