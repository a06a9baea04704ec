"""Multi-GPU orchestration of the NRRS step over torch.distributed (one process per GPU).

The wavefront queue of a bounce is split into contiguous shards, one per rank; the hash table and
the MLPs are replicated. The only exchange of the inference/decision path is the exact
normalisation sum: each rank adds its shard's 64-bit fixed-point terms into an int64
accumulator, the accumulators are all-reduced (integer SUM over NCCL/NVLink), and every rank
decides its shard against the global budget. Integer addition is exact and order-free, so the
union of the per-rank queues is bit-identical to what one GPU emits for the whole queue. Each rank
keeps its own next-bounce queue (the next bounce is sharded the same way); `queue_offsets` gives
the global position of each rank's queue when a caller wants one concatenated queue.

Every rank's context is created with the same max_queue and with sum_shards at least the world
size, so that the fixed-point shift leaves room for the terms of all shards.

Training is data-parallel: per-rank gradients (nrrs_train_grads), an all-reduce of the
gradient vector, and Adam on the mean (nrrs_adam_apply with scale 1/world).

The reference is single-GPU (one stream, no NCCL/MPI); this module has no counterpart there.
`backend` is an nrrs_b200.NRRSNetwork in production. The operations used are inferAccumulate,
decideEmitWithSum, trainGrads, copyGrads and adamApply.
"""
from __future__ import annotations


class ShardedNRRS:
    def __init__(self, backend, group=None):
        import torch.distributed as dist
        self.backend = backend
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        # the all-reduced exact sum holds world x max_queue terms: the contexts must leave room
        cfg = getattr(backend, "config", None)
        if cfg is not None and self.world > 1 and max(int(cfg.sum_shards), 1) < self.world:
            raise ValueError(f"create the contexts with sum_shards >= {self.world} (the world "
                             f"size): the all-reduced exact sum adds that many shards")

    def _allreduce(self, t):
        if self.world > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)

    def step(self, soa, rnd, n_local, budget_global, n_specular_global, params, stats, rrs,
             rrs_norm, split, queue, capacity, next_size, sum_acc, stream=0):
        """One bounce of the sharded RRS step. sum_acc: int64 tensor of one element on the
        device of this rank (zeroed here)."""
        sum_acc.zero_()
        self.backend.inferAccumulate(soa, n_local, params, stats, rrs, sum_acc, stream)
        self._allreduce(sum_acc)
        self.backend.decideEmitWithSum(rrs, rnd, n_local, budget_global, n_specular_global,
                                       sum_acc, params, rrs_norm, split, queue, capacity,
                                       next_size, stream=stream)

    def queue_offsets(self, local_size: int) -> list[int]:
        """Exclusive prefix of the per-rank next-queue sizes (all_gather of one int per rank)."""
        import torch
        dev = "cuda" if torch.cuda.is_available() and self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([local_size], dtype=torch.int64, device=dev)
        out = [torch.zeros_like(t) for _ in range(self.world)]
        if self.world > 1:
            self.dist.all_gather(out, t, group=self.group)
        else:
            out = [t]
        sizes = [int(x.item()) for x in out]
        offs, acc = [], 0
        for s in sizes:
            offs.append(acc)
            acc += s
        return offs

    def train_step(self, soa, target, n_local, grads_buf, loss=None, stream=0):
        """Data-parallel step: local gradients, all-reduce, Adam on the mean."""
        self.backend.trainGrads(soa, target, n_local, loss, stream)
        self.backend.copyGrads(grads_buf, stream)
        self._allreduce(grads_buf)
        self.backend.adamApply(grads_buf, 1.0 / self.world, stream)
