"""Row-sharded IndexBF over the ranks of a torch.distributed process group
(no counterpart in the reference, whose index lives on one device,
include/index.h:18-82).

Each rank holds a contiguous slice of the database rows on its own GPU.  A
search runs the full query batch against every shard in parallel, exchanges
the shards' [Q x k] results with one all-gather (8*Q*k bytes per shard; NCCL
over NVLink on GPUs) and merges them into the global top-k with the library's
merge kernel (ties by lower global row, as the single-index search).  Queries
are replicated: every rank passes the same queries and receives the same
results.

The local search and the merge are injectable (`local_search`, `merge`) so
that the distributed logic -- shard bases, the exchange, the merge order --
can be exercised on CPU process groups in tests; by default both are the CUDA
library's.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

import curplsh_b200 as cb


def _default_merge(dists, idxs, bases, out_idx, out_dist):
    cb.merge_shard_results(dists, idxs, bases, out_idx, out_dist, stream=torch.cuda.current_stream(dists.device))


class ShardedIndexBF:
    def __init__(self, resources, dim: int, config=None, group=None, device=None, local_search=None, merge=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.dim = int(dim)
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.index = cb.IndexBF(resources, dim, config) if local_search is None else None
        self._local_search = local_search
        self._merge = merge or _default_merge
        self.local_rows = 0
        self.bases = None

    def add(self, num: int, data) -> None:
        """Adds this rank's shard rows (collective: every rank calls it, possibly with 0 rows)."""
        if self.index is not None and num:
            self.index.add(num, data)
        self.local_rows += int(num)
        sizes = torch.tensor([self.local_rows], dtype=torch.int64, device=self.device)
        all_sizes = [torch.zeros_like(sizes) for _ in range(self.world)]
        dist.all_gather(all_sizes, sizes, group=self.group)
        self.counts = torch.cat(all_sizes)
        self.bases = torch.cumsum(self.counts, 0) - self.counts
        if int(self.counts.sum()) >= 2 ** 31:
            raise ValueError("more than 2^31 rows over all shards")

    def getNumData(self) -> int:
        return int(self.counts.sum()) if self.bases is not None else 0

    def search(self, queries, k: int, precision: int = -1):
        """Global (distances [Q, k], indices [Q, k]) on every rank (collective)."""
        Q = int(queries.shape[0])
        ld = torch.empty((Q, k), dtype=torch.float32, device=self.device)
        li = torch.empty((Q, k), dtype=torch.int32, device=self.device)
        if self._local_search is not None:
            self._local_search(queries, k, li, ld)
        else:
            # on torch's current stream, which the collective and the merge follow
            self.index.search_ex(Q, queries, k, li, ld, precision, stream=torch.cuda.current_stream(self.device))
        gd = [torch.empty((Q, k), dtype=torch.float32, device=self.device) for _ in range(self.world)]
        gi = [torch.empty((Q, k), dtype=torch.int32, device=self.device) for _ in range(self.world)]
        dist.all_gather(gd, ld, group=self.group)
        dist.all_gather(gi, li, group=self.group)
        out_d = torch.empty((Q, k), dtype=torch.float32, device=self.device)
        out_i = torch.empty((Q, k), dtype=torch.int32, device=self.device)
        self._merge(torch.stack(gd), torch.stack(gi), self.bases.to(self.device), out_i, out_d)
        return out_d, out_i

    def close(self):
        if self.index is not None:
            self.index.close()
            self.index = None
