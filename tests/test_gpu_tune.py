"""Results do not depend on the tuning knobs: every candidate value the
autotuner may pick gives the oracle's output bit for bit, and a cached CUDA
graph recorded under other knob values is re-recorded."""
import os

import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import to_dev, to_np

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def defaults_after():
    zk.load()
    zk.tune_clear()
    yield
    zk.tune_clear()
    if os.path.exists(zk.TUNE_TABLE):
        zk.tune_load(zk.TUNE_TABLE)


@pytest.mark.parametrize("knob,value", [("lde_last_logr", 9), ("lde_last_logr", 8), ("lde_last_logr", 7),
                                        ("lde_last_logr", 3), ("lde_chunk_mib", 1), ("lde_chunk_mib", 96)])
@pytest.mark.parametrize("lg,rate,cols", [(10, 3, 20), (13, 2, 33), (14, 3, 48)])
def test_lde_rows_independent_of_knobs(knob, value, lg, rate, cols):
    zk.tune_set(knob, value)
    c = O.field_data(lg * 7 + cols, cols << lg)
    rows = torch.zeros(cols << (lg + rate), dtype=torch.int64, device="cuda")
    zk.lde_rows(0, rows, to_dev(c), lg, rate, cols)
    assert np.array_equal(to_np(rows), O.lde_rows(c, lg, rate, cols))


@pytest.mark.parametrize("h", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("knob,value", [("leaf_threads", 64), ("leaf_threads", 128), ("wide_level_nodes", 1),
                                        ("wide_level_nodes", 1 << 8), ("wide_level_nodes", 1 << 40),
                                        ("coop_leaves", 0), ("coop_leaves", 1 << 40)])
def test_merkle_independent_of_knobs(h, knob, value):
    n, leaf, cap = 1 << 12, 7, 2
    zk.tune_set("%s.%d" % (knob, h), value)
    leaves = O.field_data(31 + h, n * leaf)
    n_dig, n_cap = zk.merkle_sizes(n, cap)
    dig = torch.zeros(n_dig * 4, dtype=torch.int64, device="cuda")
    caps = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
    zk.fill_digests_buf_linear_gpu(dig, caps, to_dev(leaves), n, leaf, cap, h)
    torch.cuda.synchronize()
    d, cp = O.merkle(leaves.reshape(n, leaf), leaf, cap, h)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4), d)


def test_batch_graph_rerecorded_after_knob_change():
    lg, rate, cols, cap, h = 12, 2, 32, 3, 3
    N = 1 << (lg + rate)
    c = O.field_data(77, cols << lg)
    inp = to_dev(c)
    leaves = torch.zeros(N * cols, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, cap)
    dig = torch.zeros(n_dig * 4, dtype=torch.int64, device="cuda")
    caps = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
    job = zk.commit_job(lg, rate, cols, cap, h, inp, leaves, dig, caps)
    rows = O.lde_rows(c, lg, rate, cols)
    d, cp = O.merkle(rows, cols, cap, h)
    before = zk.launch_count()
    zk.commit_batch(0, [job])
    first = zk.launch_count() - before
    before = zk.launch_count()
    zk.commit_batch(0, [job])  # same knobs: the cached graph is replayed, nothing is recorded
    assert zk.launch_count() == before
    # a knob change that alters the pass plan and the scratch size: the graph
    # cached for these exact pointers must not be replayed
    zk.tune_set("lde_last_logr", 5)
    zk.tune_set("lde_chunk_mib", 1)
    leaves.zero_()
    caps.zero_()
    before = zk.launch_count()
    zk.commit_batch(0, [job])
    assert zk.launch_count() - before > 0, "a re-recorded graph counts its launches again"
    assert first > 0
    assert np.array_equal(to_np(leaves), rows)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4), d)
