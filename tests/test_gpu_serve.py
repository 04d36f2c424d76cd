"""Continuous-batching server: every result in the mix equals the same job
committed alone, the device-memory budget is never exceeded, and jobs that do
not fit wait for memory instead of failing."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import to_dev, to_np

pytestmark = pytest.mark.gpu

SHAPES = [(12, 3, 64, 4, 0), (10, 2, 200, 3, 3), (14, 1, 33, 4, 4), (9, 3, 256, 2, 0), (13, 2, 17, 4, 1),
          (11, 3, 100, 4, 3), (15, 1, 8, 0, 0), (12, 2, 129, 4, 3)]


def alone(lg, rate, cols, cap, h, inp):
    N = 1 << (lg + rate)
    leaves = torch.zeros(N * cols, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, cap)
    dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
    caps = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
    zk.commit(0, zk.commit_job(lg, rate, cols, cap, h, inp, leaves, dig, caps))
    return to_np(caps), to_np(leaves)


@pytest.mark.parametrize("budget_mb,slots", [(4096, 8), (96, 2)])
def test_results_same_alone_and_in_the_mix(budget_mb, slots):
    inputs = [to_dev(O.field_data(700 + i, s[2] << s[0])) for i, s in enumerate(SHAPES)]
    solo = [alone(*s, inp) for s, inp in zip(SHAPES, inputs)]
    caps_host = [torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory() for s in SHAPES]
    with zk.Server(0, budget_mb << 20, slots) as srv:
        tickets = [srv.submit(*s, inp, caps_host=ch) for s, inp, ch in zip(SHAPES, inputs, caps_host)]
        for t, (caps, leaves), ch, s in zip(tickets, solo, caps_host, SHAPES):
            r = srv.wait(t)
            assert r.status == 2, r.status
            assert r.latency_ms >= r.queue_ms >= 0
            assert np.array_equal(ch.numpy().view(np.uint64), caps)
            N = 1 << (s[0] + s[1])
            got = torch.empty(N * s[2], dtype=torch.int64, device="cuda")
            # results are device pointers owned by the server: copy the leaves out
            from cuda.bindings import runtime as rt
            err, = rt.cudaMemcpy(got.data_ptr(), r.leaves, N * s[2] * 8, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
            assert err == rt.cudaError_t.cudaSuccess
            assert np.array_equal(to_np(got), leaves)
            srv.release(t)
        st = srv.stats()
        assert st["peak"] <= budget_mb << 20
        assert st["in_use"] == 0 and st["completed"] == len(SHAPES)


def test_rejects_request_larger_than_budget():
    inp = to_dev(O.field_data(1, 64 << 12))
    with zk.Server(0, 1 << 20, 2) as srv:
        with pytest.raises(zk.ZeknoxError):
            srv.submit(12, 3, 64, 4, 0, inp)


def job_bytes(lg, rate, cols, cap):
    """The server's accounting of one request's device memory: leaves,
    digests, caps and LDE scratch, each rounded up to 256 bytes."""
    N, caps = 1 << (lg + rate), 1 << cap
    t = torch.zeros(1, dtype=torch.int64)
    words = zk.commit_scratch_words(zk.commit_job(lg, rate, cols, cap, 0, t, t, t, t))
    up = lambda b: (b + 255) // 256 * 256
    return up(8 * N * cols) + up(64 * (N - caps)) + up(32 * caps) + up(8 * words)


def test_small_request_passes_a_head_that_waits_for_memory():
    big, small = (14, 3, 64, 4, 3), (10, 2, 16, 2, 3)
    budget = job_bytes(*big[:4]) * 3 // 2  # one big request at a time
    assert job_bytes(*small[:4]) <= budget // 8
    shapes = [big, big, small]
    inputs = [to_dev(O.field_data(900 + i, s[2] << s[0])) for i, s in enumerate(shapes)]
    solo = [alone(*s, inp)[0] for s, inp in zip(shapes, inputs)]
    caps_host = [torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory() for s in shapes]
    with zk.Server(0, budget, 4) as srv:
        tickets = [srv.submit(*s, inp, caps_host=ch) for s, inp, ch in zip(shapes, inputs, caps_host)]
        res = []
        for t in tickets:
            r = srv.wait(t)
            assert r.status == 2, r.status
            res.append((r.queue_ms, r.latency_ms))
            srv.release(t)
        assert srv.stats()["peak"] <= budget
    for ch, caps in zip(caps_host, solo):
        assert np.array_equal(ch.numpy().view(np.uint64), caps)
    # the small request, submitted last, started before the second big one
    # (which waited for the first one's memory)
    assert res[2][0] < res[1][0], res


@pytest.mark.parametrize("stage,status", [(zk.SERVE_FAIL_ALLOC, -2), (zk.SERVE_FAIL_SHAPE, -1),
                                          (zk.SERVE_FAIL_LAUNCH, -719)])
def test_injected_start_failure_leaves_later_requests_exact(stage, status):
    """A request whose start fails on the host (device allocation refused, a
    shape rejected when it starts, kernel queuing refused after its buffers
    were allocated) reports a negative status, gives its memory and slot back,
    and the requests after it still come out bit-exact."""
    shapes = [(11, 3, 40, 4, 0), (10, 2, 64, 3, 3), (12, 1, 24, 4, 4)]
    inputs = [to_dev(O.field_data(1200 + i, s[2] << s[0])) for i, s in enumerate(shapes)]
    solo = [alone(*s, inp)[0] for s, inp in zip(shapes, inputs)]
    caps_host = [torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory() for s in shapes]
    with zk.Server(0, 2 << 30, 2) as srv:
        srv.prepare(10, 12, 3)
        srv.prepare(10, 12, 2)
        srv.prepare(10, 12, 1)
        srv.inject_failure(stage)  # the next request the server starts: the first one
        tickets = [srv.submit(*s, inp, caps_host=ch) for s, inp, ch in zip(shapes, inputs, caps_host)]
        r = srv.wait(tickets[0])
        assert r.status == status, r.status
        assert not r.leaves and not r.caps
        srv.release(tickets[0])
        for t, ch, caps in zip(tickets[1:], caps_host[1:], solo[1:]):
            r = srv.wait(t)
            assert r.status == 2, r.status
            assert np.array_equal(ch.numpy().view(np.uint64), caps)
            srv.release(t)
        st = srv.stats()
        assert st["in_use"] == 0 and st["completed"] == len(shapes) - 1
        # the server keeps serving: the failed shape again, now without injection
        t = srv.submit(*shapes[0], inputs[0], caps_host=caps_host[0])
        assert srv.wait(t).status == 2
        assert np.array_equal(caps_host[0].numpy().view(np.uint64), solo[0])
        srv.release(t)


def test_cancel_a_queued_request():
    """One slot busy with large jobs: a small request behind them is cancelled
    while queued (status ZK_SERVE_CANCELLED, nothing counted against the
    budget), cancelling a started or finished one is refused, and the rest
    still come out bit-exact."""
    big = (16, 3, 128, 4, 0)
    small = (10, 2, 16, 2, 3)
    shapes = [big, big, small, small]
    inputs = [to_dev(O.field_data(1300 + i, s[2] << s[0])) for i, s in enumerate(shapes)]
    solo = [alone(*s, inp)[0] for s, inp in zip(shapes, inputs)]
    caps_host = [torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory() for s in shapes]
    with zk.Server(0, 8 << 30, 1) as srv:
        tickets = [srv.submit(*s, inp, caps_host=ch) for s, inp, ch in zip(shapes, inputs, caps_host)]
        srv.cancel(tickets[2])  # two large commits are ahead of it on the one slot
        r = srv.wait(tickets[2], 0.0)
        assert r.status == zk.SERVE_CANCELLED
        with pytest.raises(zk.ZeknoxError):
            srv.cancel(tickets[2])
        srv.release(tickets[2])
        for i in (0, 1, 3):
            r = srv.wait(tickets[i])
            assert r.status == 2, (i, r.status)
            assert np.array_equal(caps_host[i].numpy().view(np.uint64), solo[i])
            with pytest.raises(zk.ZeknoxError):
                srv.cancel(tickets[i])
            srv.release(tickets[i])
        st = srv.stats()
        assert st["in_use"] == 0 and st["completed"] == 3
