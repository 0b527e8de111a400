"""Document-sharded sweeps on several GPUs: one process per GPU, torch.distributed / NCCL.

EZLDA is single-GPU (EZLDA/mainKernel.cu); its sweep shards by documents because, with
iteration-start counts, a chunk's draws depend only on the global word-topic counts of the
sweep's starting topics.  Each rank keeps the whole corpus layout resident and runs the
doc-topic rebuild and the sampler for its own contiguous range of chunks.  The word side
(the word-topic rebuild and the per-word statistics) is split by word range instead:

  1. each rank rebuilds the rows of its words from the full topic array, and its words'
     share of the topic totals n_k;
  2. one all-reduce sums n_k;
  3. each rank computes its words' statistics (they read the global n_k);
  4. one all-gather moves every range's rows and statistics to every rank;
  5. each rank samples its chunks;
  6. one all-gather moves each rank's chunks' topic slice (uint16, 2 bytes per token) to
     every rank.

Randoms are keyed on the global token index, so the result is bit-identical to one GPU
with the same chunking.
"""
from __future__ import annotations

import numpy as np


def shard_words(cost: np.ndarray, world: int) -> list[tuple[int, int]]:
    """Contiguous word ranges [w0, w1), one per rank, each holding about 1/world of the
    summed per-word cost (ranges may be empty when one word outweighs a share)."""
    if world < 1:
        raise ValueError(f"cannot split words over {world} ranks")
    cost = np.asarray(cost, dtype=np.float64)
    c = np.cumsum(cost)
    total = c[-1] if len(c) else 0.0
    # a word belongs to the rank whose share holds the middle of its cost
    owner = np.minimum(world - 1, np.floor((c - cost / 2) * world / max(total, 1e-300))).astype(np.int64)
    cuts = [int(np.searchsorted(owner, r, side="left")) for r in range(world)] + [len(c)]
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


# per-word statistics: top2, k3 (uint32), phi4 (4 floats), ql (32 floats)
WORD_STAT_BYTES = 4 + 4 + 16 + 128

# Rates of the word-side time model, measured on B200: the word-topic rebuild runs at
# ~9 ps per token (0.65 ms for 71.85M tokens), and a peer copy moves 770 GB/s per direction.
REBUILD_S_PER_TOKEN = 9.0e-12
LINK_BYTES_PER_S = 770e9


def word_bytes(num_words: int, num_dense: int, K: int, sparse_slot: np.ndarray, qtab_rounds: int = 0) -> np.ndarray:
    """Bytes each word adds to the word-side all-gather: its dense row (4K, plus its Q-round
    table of 32 x qtab_rounds float pairs) or its sparse slot plus row length (4 per entry,
    4), and its statistics."""
    b = np.empty(num_words, dtype=np.float64)
    b[:num_dense] = 4 * K + 256 * qtab_rounds
    b[num_dense:] = 4 * (np.asarray(sparse_slot, dtype=np.float64) + 1)
    return b + WORD_STAT_BYTES


def word_ranges(word_tokens: np.ndarray, num_dense: int, K: int, sparse_slot: np.ndarray, world: int,
                s_per_token: float = REBUILD_S_PER_TOKEN, link_bps: float = LINK_BYTES_PER_S, qtab_rounds: int = 0):
    """Contiguous word ranges, one per rank, for the word side.  A rank's word-side time is
    modelled as its rebuild (tokens x s_per_token) plus the all-gather, whose segments
    are all as large as the largest range's bytes ((world - 1) segments received at
    link_bps).  The ranges balance tokens/total + lam * bytes/total; lam is scanned and the
    split with the smallest modelled max(rebuild) + all-gather is returned, with that time
    in seconds."""
    tok = np.asarray(word_tokens, dtype=np.float64)
    byt = word_bytes(len(tok), num_dense, K, sparse_slot, qtab_rounds)
    ct = np.concatenate([[0.0], np.cumsum(tok)])
    cb = np.concatenate([[0.0], np.cumsum(byt)])
    best, best_t = None, np.inf
    for lam in [0.0] + list(np.geomspace(1e-3, 1e3, 31)) + [np.inf]:
        cost = byt / max(byt.sum(), 1.0) if lam == np.inf else tok / max(tok.sum(), 1.0) + lam * byt / max(byt.sum(), 1.0)
        r = shard_words(cost, world)
        t_tok = max(ct[b] - ct[a] for a, b in r) * s_per_token
        t_net = (world - 1) * max(cb[b] - cb[a] for a, b in r) / link_bps
        if t_tok + t_net < best_t:
            best, best_t = r, t_tok + t_net
    return best, best_t


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
        if len(self.slices) == 1:
            return
        a, b = self.slices[self.rank]
        self.send[:b - a].copy_(self.t[a:b])
        dist.all_gather_into_tensor(self.recv, self.send, group=self.group)
        for r, (a, b) in enumerate(self.slices):
            if r != self.rank and b > a:
                self.t[a:b].copy_(self.recv[r * self.seg:r * self.seg + (b - a)])


class WordExchange:
    """Moves every rank's word range of the word side to every rank.  The word side is a
    dict of flat byte tensors (the trainer's device arrays, or CPU tensors with gloo):
    "dense" (K int32 per dense word), "sparse_ent" (fixed slots, sparse_off[s] the first
    entry of sparse word s), "sparse_nnz", "top2", "k3", "phi4", "ql", plus the int32
    "n_k", and above 2048 topics "qtab" (each dense word's Q-round table, qtab_bytes per
    dense word).  A rank's range is a handful of contiguous byte pieces; they are packed into an
    equal-sized send segment (padded to the largest range's, 16-byte aligned), one
    all-gather brings every segment, and the other ranks' pieces are copied into place."""

    FIELDS = ("dense", "sparse_ent", "sparse_nnz", "top2", "k3", "phi4", "ql", "qtab")
    PER_WORD = {"top2": 4, "k3": 4, "phi4": 16, "ql": 128}

    def __init__(self, side, K: int, num_dense: int, sparse_off: np.ndarray, ranges, group=None, qtab_bytes: int = 0):
        import torch
        import torch.distributed as dist
        self.side, self.ranges, self.group = side, ranges, group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        V = len(sparse_off) - 1 + num_dense
        off = np.asarray(sparse_off, dtype=np.int64)
        self.pieces = []
        for w0, w1 in ranges:
            if not (0 <= w0 <= w1 <= V):
                raise ValueError(f"word range [{w0}, {w1}) outside [0, {V})")
            d0, d1 = min(w0, num_dense), min(w1, num_dense)
            s0, s1 = max(w0, num_dense) - num_dense, max(w1, num_dense) - num_dense
            p = [("dense", 4 * K * d0, 4 * K * (d1 - d0)),
                 ("sparse_ent", 4 * int(off[s0]), 4 * int(off[s1] - off[s0])),
                 ("sparse_nnz", 4 * s0, 4 * (s1 - s0)),
                 ("qtab", qtab_bytes * d0, qtab_bytes * (d1 - d0))]
            p += [(f, b * w0, b * (w1 - w0)) for f, b in self.PER_WORD.items()]
            self.pieces.append([x for x in p if x[2] > 0])
        self.seg = max(16, max(sum(n for _, _, n in p) for p in self.pieces))
        self.seg = (self.seg + 15) & ~15
        dev = side["n_k"].device
        self.send = torch.zeros(self.seg, dtype=torch.uint8, device=dev)
        self.recv = torch.empty(len(ranges) * self.seg, dtype=torch.uint8, device=dev)

    @property
    def bytes_per_rank(self) -> int:
        return self.seg

    def pack(self, rank: int | None = None, out=None):
        """Copies `rank`'s pieces (default: this rank's) into a send segment."""
        out = self.send if out is None else out
        pos = 0
        for f, a, n in self.pieces[self.rank if rank is None else rank]:
            out[pos:pos + n].copy_(self.side[f][a:a + n])
            pos += n
        return out

    def unpack(self, recv, skip: int | None = None) -> None:
        """Copies every rank's pieces but `skip`'s (default: this rank's) out of the
        gathered segments."""
        skip = self.rank if skip is None else skip
        for r, pieces in enumerate(self.pieces):
            if r == skip:
                continue
            pos = r * self.seg
            for f, a, n in pieces:
                self.side[f][a:a + n].copy_(recv[pos:pos + n])
                pos += n

    def reduce_totals(self) -> None:
        """Sums n_k over the ranks (each rank's n_k holds its words' tokens only)."""
        import torch.distributed as dist
        dist.all_reduce(self.side["n_k"], group=self.group)

    def exchange(self) -> None:
        import torch.distributed as dist
        self.pack()
        dist.all_gather_into_tensor(self.recv, self.send, group=self.group)
        self.unpack(self.recv)


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


def word_side_tensors(trainer, device: int):
    """Zero-copy torch views of the trainer's word side: flat uint8 tensors for
    WordExchange's fields, an int32 tensor for n_k, and the host copy of the sparse slot
    offsets (sparse_off plus the capacity at the end)."""
    import torch
    ws = trainer.word_side()
    dev = torch.device("cuda", device)
    V, Vd, K = ws.vocab, ws.num_dense, ws.K

    def view(ptr, n, typestr="|u1"):
        return torch.as_tensor(_CudaArray(ptr or 0, n, typestr), device=dev) if n > 0 else \
            torch.empty(0, dtype=torch.uint8 if typestr == "|u1" else torch.int32, device=dev)

    off = np.empty(V - Vd + 1, dtype=np.int64)
    if V > Vd:
        off[:-1] = view(ws.sparse_off, V - Vd, "<u4").cpu().numpy()
    off[-1] = ws.sparse_capacity
    side = {"n_k": view(ws.n_k, K, "<i4"), "dense": view(ws.dense_wt, 4 * K * Vd),
            "sparse_ent": view(ws.sparse_ent, 4 * ws.sparse_capacity), "sparse_nnz": view(ws.sparse_nnz, 4 * (V - Vd)),
            "top2": view(ws.top2, 4 * V), "k3": view(ws.k3, 4 * V), "phi4": view(ws.phi4, 16 * V),
            "ql": view(ws.ql, 128 * V), "qtab": view(ws.qtab, 256 * ws.qtab_rounds * Vd)}
    return side, off


class ShardedTrainer:
    """A Trainer that rebuilds the word side of its rank's word range, samples its rank's
    chunks, and exchanges both with the other ranks every sweep."""

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
        side, off = word_side_tensors(self.tr, device)
        ws = self.tr.word_side()
        self.word_ranges, self.word_side_s = word_ranges(corpus.word_count(), ws.num_dense, K, np.diff(off), world,
                                                         qtab_rounds=ws.qtab_rounds)
        self.tr.set_word_range(*self.word_ranges[rank])
        self.wx = WordExchange(side, K, ws.num_dense, off, self.word_ranges, group, qtab_bytes=256 * ws.qtab_rounds)
        self.group = group
        self.device = device

    @property
    def own_slice(self) -> tuple[int, int]:
        a, b = self.ranges[self.rank]
        return int(self.chunk_tok[a]), int(self.chunk_tok[b])

    def sweep(self, ll: bool = False) -> None:
        """One sweep from the topics every rank holds, leaving new topics in this rank's
        chunks only: the word side of this rank's words, the n_k all-reduce, the word
        statistics, the word-side all-gather, then this rank's chunks."""
        self.tr.update_wt()
        if self.world > 1:
            self.wx.reduce_totals()
        self.tr.max_topic()
        if self.world > 1:
            self.wx.exchange()
        self.tr.sweep_chunks(ll=ll)

    def iterate(self, n: int = 1, ll: bool = False) -> float | None:
        """n sweeps, each followed by the topic all-gather; with ll=True the global mean
        per-token log-likelihood of the last."""
        import torch
        import torch.distributed as dist
        for _ in range(n):
            self.sweep(ll=ll)
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
