"""Document-sharded sweeps on several GPUs: one process per GPU, torch.distributed / NCCL.

EZLDA is single-GPU (EZLDA/mainKernel.cu); its sweep shards by documents because, with
iteration-start counts, a chunk's draws depend only on the global word-topic counts of the
sweep's starting topics.  Each rank keeps the whole corpus layout resident, rebuilds the
word-topic counts from the full topic array (replicated, ~0.8 ms for 72M tokens), and runs
the doc-topic rebuild and the sampler for its own contiguous range of chunks.  After every
sweep one all-gather moves each rank's chunks' topic slice (uint16, 2 bytes per token) to
every rank, which is the only exchange.  Randoms are keyed on the global token index, so the result is
bit-identical to one GPU with the same chunking.
"""
from __future__ import annotations

import numpy as np


def shard_chunks(num_chunks: int, world: int) -> list[tuple[int, int]]:
    """Contiguous, as-even-as-possible chunk ranges, one per rank."""
    if world < 1 or num_chunks < world:
        raise ValueError(f"{num_chunks} chunks cannot be split over {world} ranks")
    return [(r * num_chunks // world, (r + 1) * num_chunks // world) for r in range(world)]


class TopicExchange:
    """After a sweep each rank holds new topics only for its own chunks' tokens, one
    contiguous slice [chunk_tok[first], chunk_tok[last]) of the word-sorted 16-bit topic
    array.  One all-gather moves every slice to every rank: each rank's slice is copied
    into an equal-sized send segment (padded to the longest slice), the segments are
    gathered into one buffer, and the other ranks' slices are copied into place.  Neither
    NCCL nor gloo has a 16-bit integer type, so the slices travel as bytes.  Works on CUDA
    tensors with NCCL and on CPU tensors with gloo."""

    def __init__(self, topics, chunk_tok, ranges, group=None):
        import torch
        import torch.distributed as dist
        self.t = topics.view(torch.uint8)
        self.slices = [(2 * int(chunk_tok[a]), 2 * int(chunk_tok[b])) for a, b in ranges]
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.seg = max(1, max(b - a for a, b in self.slices))
        self.seg = (self.seg + 15) & ~15  # 16-byte segments
        self.send = torch.zeros(self.seg, dtype=torch.uint8, device=topics.device)
        self.recv = torch.empty(len(ranges) * self.seg, dtype=torch.uint8, device=topics.device)

    def exchange(self) -> None:
        import torch.distributed as dist
        a, b = self.slices[self.rank]
        self.send[:b - a].copy_(self.t[a:b])
        dist.all_gather_into_tensor(self.recv, self.send, group=self.group)
        for r, (a, b) in enumerate(self.slices):
            if r != self.rank and b > a:
                self.t[a:b].copy_(self.recv[r * self.seg:r * self.seg + (b - a)])


class _CudaArray:
    """__cuda_array_interface__ view of a device buffer owned by the library."""

    def __init__(self, ptr: int, n: int, typestr: str = "<i2"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def topics_tensor(trainer, device: int):
    """Zero-copy int16 torch view of the trainer's uint16 topic array."""
    import torch
    ptr, n = trainer.topics_device()
    return torch.as_tensor(_CudaArray(ptr, n), device=torch.device("cuda", device))


class ShardedTrainer:
    """A Trainer that samples its rank's chunks and exchanges topics after each sweep."""

    def __init__(self, corpus, K: int, rank: int, world: int, device: int, group=None, **kw):
        import torch
        from . import Trainer
        self.rank, self.world = rank, world
        self.tr = Trainer(corpus, K=K, device=device, **kw)
        self.tr.set_stream(torch.cuda.current_stream(device).cuda_stream)
        self.ranges = shard_chunks(corpus.info.num_chunks, world)
        self.tr.set_chunk_range(*self.ranges[rank])
        self.z = topics_tensor(self.tr, device)
        self.chunk_tok = corpus.chunk_tok()
        self.ex = TopicExchange(self.z, self.chunk_tok, self.ranges, group)
        self.group = group
        self.device = device

    @property
    def own_slice(self) -> tuple[int, int]:
        a, b = self.ranges[self.rank]
        return int(self.chunk_tok[a]), int(self.chunk_tok[b])

    def iterate(self, n: int = 1, ll: bool = False) -> float | None:
        """n sweeps; with ll=True the global mean per-token log-likelihood of the last."""
        import torch
        import torch.distributed as dist
        for _ in range(n):
            self.tr.iterate(1, ll=ll)
            self.ex.exchange()
        if ll and n > 0:
            s, t = self.tr.loglik()
            v = torch.tensor([s, float(t)], dtype=torch.float64, device=torch.device("cuda", self.device))
            dist.all_reduce(v, group=self.group)
            return float(v[0] / v[1])
        return None

    def topics(self) -> np.ndarray:
        return self.tr.topics()

    def close(self) -> None:
        self.tr.close()
