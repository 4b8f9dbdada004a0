"""Row-sharded search over a 2-rank gloo process group on CPU: the shard
bases, the all-gather exchange and the merge order must give the same top-k
as one search over the whole database.  The local searches here are the FP64
oracle and the merge a numpy restatement of the library's merge rule (lower
global row first on equal distances); the CUDA merge kernel itself is tested
on the GPU (test_gpu_sharded.py)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle

N, Q, D, K = 3001, 23, 16, 10


def _data():
    rng = np.random.default_rng(77)
    base = rng.integers(0, 4, size=(N, D)).astype(np.float32)  # many exact ties
    queries = rng.integers(0, 4, size=(Q, D)).astype(np.float32)
    return base, queries


def numpy_merge(dists, idxs, bases, out_idx, out_dist):
    """Lexicographic (distance, global row) merge of [G, Q, k] shard results."""
    G, Qn, k = dists.shape
    for q in range(Qn):
        cand = []
        for s in range(G):
            for j in range(k):
                li = int(idxs[s, q, j])
                if li >= 0:
                    cand.append((float(dists[s, q, j]), int(bases[s]) + li))
        cand.sort()
        for t in range(k):
            if t < len(cand):
                out_dist[q, t] = cand[t][0]
                out_idx[q, t] = cand[t][1]
            else:
                out_dist[q, t] = np.finfo(np.float32).max
                out_idx[q, t] = -1


def _worker(rank, world, port, outdir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from curplsh_b200.sharded import ShardedIndexBF
    base, queries = _data()
    cuts = [0, 1234, N] if world == 2 else [0, N]
    shard = base[cuts[rank]:cuts[rank + 1]]

    def local_search(q, k, li, ld):
        d, i = oracle.knn(shard, q.numpy(), k)
        ld.copy_(torch.from_numpy(d.astype(np.float32)))
        li.copy_(torch.from_numpy(i.astype(np.int32)))

    def merge(gd, gi, bases, out_i, out_d):
        oi = np.empty(tuple(out_i.shape), np.int32)
        od = np.empty(tuple(out_d.shape), np.float32)
        numpy_merge(gd.numpy(), gi.numpy(), bases.numpy(), oi, od)
        out_i.copy_(torch.from_numpy(oi))
        out_d.copy_(torch.from_numpy(od))

    ix = ShardedIndexBF(None, D, device=torch.device("cpu"), local_search=local_search, merge=merge)
    ix.add(shard.shape[0], shard)
    assert ix.getNumData() == N
    d, i = ix.search(torch.from_numpy(queries), K)
    np.savez(os.path.join(outdir, f"rank{rank}.npz"), d=d.numpy(), i=i.numpy())
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_sharded_search_equals_single_search(tmp_path):
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    base, queries = _data()
    rd, ri = oracle.knn(base, queries, K)
    for r in range(2):
        f = np.load(tmp_path / f"rank{r}.npz")
        d, i = f["d"], f["i"]
        np.testing.assert_array_equal(i, ri, err_msg=f"rank {r}: indices")
        np.testing.assert_allclose(d, rd.astype(np.float32), rtol=0, atol=0, err_msg=f"rank {r}: distances")


def test_numpy_merge_handles_padding():
    d = np.full((2, 1, 3), np.finfo(np.float32).max, np.float32)
    i = np.full((2, 1, 3), -1, np.int32)
    d[0, 0, 0], i[0, 0, 0] = 5.0, 2
    d[1, 0, 0], i[1, 0, 0] = 5.0, 0
    oi = np.empty((1, 3), np.int32)
    od = np.empty((1, 3), np.float32)
    numpy_merge(d, i, np.array([0, 10]), oi, od)
    assert oi.tolist() == [[2, 10, -1]]
