"""Ad-range shards: each shard (one per GPU, or several on one GPU) holds the
postings whose ad ids fall in its slice [lo, hi) of the ad space, with ids
rebased to the slice. A query runs on every shard against the same terms; the
shards' bitmaps are disjoint word ranges of the full bitmap, and the full id
list is the shards' id lists in shard order, each shifted by its lo. Nothing
has to be combined bit by bit (term sharding would need a bitwise-OR reduce,
which NCCL does not have).

Slices start at multiples of SLICE_ALIGN ads, so every slice begins on a
16-byte boundary of the full bitmap row and a shard can write its words in
place (its batch writes exactly the words of its own n_ads).

The reference is single-GPU; this module has no reference counterpart.
"""
from __future__ import annotations

import numpy as np

SLICE_ALIGN = 4096  # ads: 128 words, so slices start 16-byte aligned in a row


def ad_slices(n_ads: int, world: int) -> list[tuple[int, int]]:
    """[lo, hi) ad ranges of `world` shards, lo a multiple of SLICE_ALIGN,
    covering [0, n_ads) in order (trailing shards may be empty)."""
    if world <= 0 or n_ads < 0:
        raise ValueError("bad n_ads/world")
    units = -(-n_ads // SLICE_ALIGN)
    base, extra = divmod(units, world)
    out, u = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        lo, hi = min(u * SLICE_ALIGN, n_ads), min((u + n) * SLICE_ALIGN, n_ads)
        out.append((lo, hi))
        u += n
    return out


def shard_csr(offsets: np.ndarray, ads: np.ndarray, lo: int, hi: int):
    """CSR lists restricted to ads in [lo, hi), ids rebased to lo (lists stay
    sorted; every term keeps its slot, possibly empty)."""
    off = np.asarray(offsets, dtype=np.uint64)
    a = np.asarray(ads, dtype=np.uint32)
    keep = (a >= lo) & (a < hi)
    term = np.repeat(np.arange(off.size - 1, dtype=np.int64), np.diff(off).astype(np.int64))
    cnt = np.bincount(term[keep], minlength=off.size - 1).astype(np.uint64)
    new_off = np.zeros(off.size, dtype=np.uint64)
    np.cumsum(cnt, out=new_off[1:])
    return new_off, (a[keep] - np.uint32(lo)).astype(np.uint32)


class AdRangeShards:
    """Shards of one index on the devices given (one shard per entry of
    `devices`; the same device may appear more than once). Build from CSR
    lists over the full ad space."""

    def __init__(self, offsets, ads, n_terms: int, n_ads: int, devices, **index_kw):
        from .index import Index
        self.n_terms, self.n_ads = n_terms, n_ads
        self.slices = ad_slices(n_ads, len(devices))
        self.devices = list(devices)
        self.indexes = []
        for (lo, hi), dev in zip(self.slices, self.devices):
            so, sa = shard_csr(offsets, ads, lo, hi)
            self.indexes.append(Index.from_csr(so, sa, n_terms, max(hi - lo, 1), device=dev, **index_kw)
                                if hi > lo else None)

    def batch_run(self, workspaces, d_terms, d_offsets, n_queries: int, d_bitmaps, stride_words: int, **kw):
        """Bitmaps of n_queries queries over the full ad space into d_bitmaps
        (n_queries x stride_words words, on the shards' device): each shard
        writes its own word range. workspaces: one per non-empty shard."""
        wi = 0
        for (lo, hi), ix in zip(self.slices, self.indexes):
            if ix is None:
                continue
            ix.batch_run(workspaces[wi], d_terms, d_offsets, n_queries, d_bitmaps[:, lo // 32:], stride_words, **kw)
            wi += 1

    def workspaces(self, max_queries: int, max_terms: int):
        return [ix.workspace(max_queries, max_terms) for ix in self.indexes if ix is not None]

    def free(self):
        for ix in self.indexes:
            if ix is not None:
                ix.free()
        self.indexes = []


def merge_ids(parts: list[np.ndarray], slices: list[tuple[int, int]]) -> np.ndarray:
    """One query's full id list from its per-shard lists (shard order)."""
    return np.concatenate([np.asarray(p, dtype=np.uint64) + lo for p, (lo, _) in zip(parts, slices)]
                          ).astype(np.uint32) if parts else np.zeros(0, np.uint32)


def gather_bitmap_slices(local: "torch.Tensor", n_words: int, slices, dist) -> "torch.Tensor":  # noqa: F821
    """Full bitmaps (n_q x n_words words) on every rank from each rank's slice
    (n_q x its slice's words, rank = shard): one all-gather of equal-size
    padded slices over the process group (NCCL over NVLink on GPUs, gloo on
    the host), then the rows are reassembled."""
    import torch
    world = dist.get_world_size()
    n_q = local.shape[0]
    wmax = max(max(-(-(hi - lo) // 32) for lo, hi in slices), 1)
    pad = torch.zeros((n_q, wmax), dtype=local.dtype, device=local.device)
    pad[:, :local.shape[1]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad)
    out = torch.zeros((n_q, n_words), dtype=local.dtype, device=local.device)
    for r, (lo, hi) in enumerate(slices):
        w = -(-(hi - lo) // 32)
        out[:, lo // 32:lo // 32 + w] = bufs[r][:, :w]
    return out
