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
    try:
        import torch.distributed._symmetric_memory as symm_mem  # noqa: F401
    except Exception as e:  # pragma: no cover
        pytest.skip("no symmetric memory: %s" % e)
    n = 1 << lg
    c = O.field_data(17 * lg + cols, cols * n)
    caps, dig, leaves = zd.commit_distributed_p2p(to_dev(c), lg, rate, cols, cap, h)
    rows = O.lde_rows(c, lg, rate, cols)
    d, cp = O.merkle(rows, cols, cap, h)
    assert np.array_equal(to_np(leaves), np.ascontiguousarray(rows).reshape(-1))
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4), d)
