"""The distributed commit (zeknox_b200.dist) across gloo ranks on CPU.

Every rank extends its shard of the columns (the oracle's LDE stands in for
the GPU stage), the real exchange and row assembly of
``dist.commit_sharded`` move the rows with ``all_to_all_single``, and each
hashing rank builds its subtrees with the library's exported CPU Merkle
builder; the caps, the digest ranges and the leaf rows must equal the
single-process commitment bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from zeknox_b200 import multi


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, case, result):
    import zeknox_b200 as zk
    from oracle import oracle as O
    from zeknox_b200 import dist as zd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lg, rate, cols, cap_h, h = case
        n, N = 1 << lg, 1 << (lg + rate)
        coeffs = O.field_data(900 + cols, cols * n)
        c0, k = multi.split_columns(cols, world)[rank]
        mine = torch.from_numpy(coeffs[c0 * n:(c0 + k) * n].view(np.int64).copy())

        def lde(c, kk):
            rows = O.lde_rows(c.numpy().view(np.uint64), lg, rate, kk)
            return torch.from_numpy(np.ascontiguousarray(rows).reshape(-1).view(np.int64).copy())

        def merkle(leaves, n_leaves, leaf_size, hh):
            nd, nc = zk.merkle_sizes(n_leaves, hh)
            dg = torch.zeros(max(nd, 1) * 4, dtype=torch.int64)
            cp = torch.zeros(nc * 4, dtype=torch.int64)
            zk.fill_digests_buf_linear_cpu(dg, cp, leaves, n_leaves, leaf_size, hh, h)
            return dg[:nd * 4], cp

        caps, digests, leaves = zd.commit_sharded(mine, lg, rate, cols, cap_h, lde, merkle)
        rows_full = np.ascontiguousarray(O.lde_rows(coeffs, lg, rate, cols)).reshape(-1)
        d_full, c_full = O.merkle(rows_full, cols, cap_h, h)
        ok = np.array_equal(caps.numpy().view(np.uint64).reshape(-1, 4), c_full)
        G = multi.merkle_gpus(1 << cap_h, world)
        if rank < G:
            rows_per = N // G
            caps_g = (1 << cap_h) // G
            D = 2 * (N // (1 << cap_h)) - 2
            ok &= np.array_equal(leaves.numpy().view(np.uint64), rows_full[rank * rows_per * cols:(rank + 1) * rows_per * cols])
            ok &= np.array_equal(digests.numpy().view(np.uint64).reshape(-1, 4),
                                 d_full[rank * caps_g * D:(rank + 1) * caps_g * D])
        else:
            ok &= digests is None and leaves is None
        res = [None] * world
        dist.all_gather_object(res, bool(ok))
        if rank == 0:
            result.put(all(res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case", [
    (2, (5, 2, 7, 2, 3)),   # two hashing ranks, uneven columns
    (3, (4, 3, 5, 2, 0)),   # 3 ranks, 2 of them hash (power of two)
    (3, (6, 1, 2, 1, 4)),   # more ranks than columns: rank 2 extends nothing
    (4, (5, 1, 9, 0, 3)),   # one cap: only rank 0 hashes
    (2, (3, 1, 4, 4, 3)),   # caps == leaves: subtrees of one leaf
])
def test_distributed_commit_equals_single_process(world, case):
    ctx = mp.get_context("spawn")
    result = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, result)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0] * world, codes
    assert result.get(timeout=5) is True
