"""The distributed commit on the GPU through NCCL (a one-rank process group:
this pool gives one GPU per run; the multi-rank exchange is covered by the
gloo tests in test_dist_host.py).  The result must equal zeknox_commit's."""
import datetime

import numpy as np
import pytest
import torch
import torch.distributed as dist

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import to_dev, to_np
from zeknox_b200 import dist as zd
from zeknox_b200 import multi

pytestmark = pytest.mark.gpu


@pytest.fixture
def nccl_group():
    if dist.is_initialized():
        pytest.skip("a process group already exists")
    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    yield
    dist.destroy_process_group()


@pytest.mark.parametrize("lg,rate,cols,cap,h", [(10, 2, 24, 3, 3), (12, 3, 16, 4, 0), (8, 1, 5, 0, 4)])
def test_distributed_commit_one_rank_nccl(nccl_group, lg, rate, cols, cap, h):
    n, N = 1 << lg, 1 << (lg + rate)
    c = O.field_data(31 * lg + cols, cols * n)
    caps, dig, leaves = zd.commit_distributed(to_dev(c), lg, rate, cols, cap, h)
    torch.cuda.synchronize()
    rows = O.lde_rows(c, lg, rate, cols)
    d, cp = O.merkle(rows, cols, cap, h)
    assert np.array_equal(to_np(leaves), np.ascontiguousarray(rows).reshape(-1))
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4), d)


@pytest.mark.parametrize("lg,rate,cols,cap,h", [(10, 2, 24, 3, 3), (12, 3, 16, 4, 0)])
def test_distributed_commit_p2p_one_rank(nccl_group, lg, rate, cols, cap, h):
    n = 1 << lg
    c = O.field_data(17 * lg + cols, cols * n)
    caps, dig, leaves = zd.commit_distributed_p2p(to_dev(c), lg, rate, cols, cap, h)
    rows = O.lde_rows(c, lg, rate, cols)
    d, cp = O.merkle(rows, cols, cap, h)
    assert np.array_equal(to_np(leaves), np.ascontiguousarray(rows).reshape(-1))
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4), d)


def _p2p_rank(rank, world, port, lg, rate, cols, cap, h, out_dir):
    import os
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 1 << lg
        c = O.field_data(23 * lg + cols, cols * n)
        c0, k = zd.split_columns(cols, world)[rank]
        caps, dig, leaves = zd.commit_distributed_p2p(to_dev(c[c0 * n:(c0 + k) * n]), lg, rate, cols, cap, h)
        np.save(os.path.join(out_dir, "caps%d.npy" % rank), to_np(caps))
        if dig is not None:
            np.save(os.path.join(out_dir, "dig%d.npy" % rank), to_np(dig))
            np.save(os.path.join(out_dir, "leaves%d.npy" % rank), to_np(leaves))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("lg,rate,cols,cap,h", [(10, 2, 24, 3, 3), (9, 3, 7, 1, 0)])
def test_distributed_commit_p2p_two_ranks_ipc(tmp_path, lg, rate, cols, cap, h):
    """Two ranks (processes) on the one GPU of this run, host barriers over
    gloo: each rank maps the other's row shard through its CUDA IPC handle and
    the scatter kernels store into both shards; no kernel waits on another
    rank.  The assembled shards must be the single-process commitment."""
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_p2p_rank, args=(2, port, lg, rate, cols, cap, h, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    n, N = 1 << lg, 1 << (lg + rate)
    c = O.field_data(23 * lg + cols, cols * n)
    rows = O.lde_rows(c, lg, rate, cols)
    d, cp = O.merkle(rows, cols, cap, h)
    G = zd.merkle_gpus(1 << cap, 2)
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / ("caps%d.npy" % r)).reshape(-1, 4), cp)
    shards = multi.split_subtrees(N, 1 << cap, 2)
    for r in range(G):
        sh = shards[r]
        l0, ln = sh["leaves"]
        d0, dn = sh["digests"]
        assert np.array_equal(np.load(tmp_path / ("leaves%d.npy" % r)), rows.reshape(N, cols)[l0:l0 + ln].reshape(-1))
        assert np.array_equal(np.load(tmp_path / ("dig%d.npy" % r)).reshape(-1, 4), d[d0:d0 + dn])
