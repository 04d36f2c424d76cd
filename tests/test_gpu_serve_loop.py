"""Device-resident request loop (zeknox_server_create_ex with
ZK_SERVE_DEVICE_LOOP): every request's leaves, digests and caps equal the
same job committed alone through zeknox_commit, from coefficients and from
evaluations; a request whose bounded wait runs out fails alone; the loop
exits when idle and comes back."""
import time

import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import to_dev, to_np

pytestmark = pytest.mark.gpu

# (lg_n, rate, cols, cap, hash): cooperative and one-per-thread leaves, wide
# levels (2^16 leaves and more), caps written by the fold (subtrees of <= 64
# leaves) and by the tail, one cap, two and three passes per column chunk,
# three column chunks (2^22 rows: 16 columns a chunk), ragged column counts
SHAPES = [(9, 1, 16, 4, 0), (10, 3, 33, 0, 3), (12, 2, 64, 4, 0), (13, 3, 24, 4, 3), (11, 1, 100, 2, 0),
          (19, 3, 40, 4, 0), (19, 1, 8, 3, 3), (9, 3, 7, 4, 3), (14, 2, 17, 1, 0),
          # the hashes without a cooperative form: one permutation per thread
          # in the fold and tail (Keccak 1, Poseidon-BN128 2, Monolith 4)
          (12, 3, 17, 4, 1), (10, 1, 5, 0, 1), (9, 1, 12, 2, 2), (13, 2, 30, 4, 4), (10, 3, 9, 0, 4)]


def alone(lg, rate, cols, cap, h, inp):
    N = 1 << (lg + rate)
    leaves = torch.zeros(N * cols, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, cap)
    dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
    caps = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
    zk.commit(0, zk.commit_job(lg, rate, cols, cap, h, inp, leaves, dig, caps))
    return to_np(leaves), to_np(dig)[: n_dig * 4], to_np(caps)


def device_words(ptr, words):
    from cuda.bindings import runtime as rt
    out = torch.empty(max(words, 1), dtype=torch.int64, device="cuda")
    if words:
        err, = rt.cudaMemcpy(out.data_ptr(), ptr, words * 8, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
        assert err == rt.cudaError_t.cudaSuccess
    return to_np(out)[:words]


def check(srv, t, shape, solo, caps_host):
    lg, rate, cols, cap, h = shape
    r = srv.wait(t)
    assert r.status == 2, r.status
    N = 1 << (lg + rate)
    n_dig, _ = zk.merkle_sizes(N, cap)
    leaves, dig, caps = solo
    assert np.array_equal(caps_host.numpy().view(np.uint64), caps)
    assert np.array_equal(device_words(r.leaves, N * cols), leaves)
    assert np.array_equal(device_words(r.digests, n_dig * 4), dig)
    srv.release(t)


def test_results_same_as_alone():
    inputs = [to_dev(O.field_data(4100 + i, s[2] << s[0])) for i, s in enumerate(SHAPES)]
    # one request reads its coefficients from pinned host memory
    inputs[2] = inputs[2].cpu().pin_memory()
    solo = [alone(*s, inp.cuda()) for s, inp in zip(SHAPES, inputs)]
    caps_host = [torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory() for s in SHAPES]
    with zk.Server(0, 8 << 30, 16, device_loop=True) as srv:
        tickets = [srv.submit(*s, inp, caps_host=ch) for s, inp, ch in zip(SHAPES, inputs, caps_host)]
        for t, s, so, ch in zip(tickets, SHAPES, solo, caps_host):
            check(srv, t, s, so, ch)
        st = srv.stats()
        assert st["in_use"] == 0 and st["completed"] == len(SHAPES)


# evaluation-form inputs: the loop runs the inverse transform first (copy,
# inverse passes of 1-3 per column, bit-reversal reorder); 2^9 .. 2^20 points
# (single passes of 2^9 .. 2^12, two and three passes), one from pinned host
# memory
VALUE_SHAPES = [(9, 1, 16, 4, 0), (12, 2, 33, 3, 3), (14, 3, 20, 4, 0), (17, 1, 8, 2, 3), (20, 1, 4, 4, 0),
                (11, 3, 12, 0, 1)]


def test_evaluation_inputs_same_as_alone():
    inputs = [to_dev(O.field_data(4700 + i, s[2] << s[0])) for i, s in enumerate(VALUE_SHAPES)]
    inputs[1] = inputs[1].cpu().pin_memory()
    solo = []
    for s, inp in zip(VALUE_SHAPES, inputs):
        lg, rate, cols, cap, h = s
        N = 1 << (lg + rate)
        leaves = torch.zeros(N * cols, dtype=torch.int64, device="cuda")
        n_dig, n_cap = zk.merkle_sizes(N, cap)
        dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
        caps = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
        zk.commit(0, zk.commit_job(lg, rate, cols, cap, h, inp.cuda(), leaves, dig, caps, input_is_values=True))
        solo.append((to_np(leaves), to_np(dig)[: n_dig * 4], to_np(caps)))
    caps_host = [torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory() for s in VALUE_SHAPES]
    with zk.Server(0, 4 << 30, 8, device_loop=True) as srv:
        tickets = [srv.submit(*s, inp, caps_host=ch, input_is_values=True)
                   for s, inp, ch in zip(VALUE_SHAPES, inputs, caps_host)]
        for t, s, so, ch in zip(tickets, VALUE_SHAPES, solo, caps_host):
            check(srv, t, s, so, ch)
        # and a coefficient-form request after them, through the same loop
        shape = (13, 3, 24, 4, 3)
        inp = to_dev(O.field_data(4790, shape[2] << shape[0]))
        ch = torch.zeros((1 << shape[3]) * 4, dtype=torch.int64).pin_memory()
        check(srv, srv.submit(*shape, inp, caps_host=ch), shape, alone(*shape, inp), ch)


def test_more_requests_than_ring_entries():
    shapes = [(9 + i % 4, 1 + i % 3, 8 + 5 * i, i % 5, (0, 3)[i % 2]) for i in range(40)]
    inputs = [to_dev(O.field_data(4300 + i, s[2] << s[0])) for i, s in enumerate(shapes)]
    solo = [alone(*s, inp) for s, inp in zip(shapes, inputs)]
    caps_host = [torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory() for s in shapes]
    with zk.Server(0, 2 << 30, 16, device_loop=True) as srv:
        tickets = [srv.submit(*s, inp, caps_host=ch) for s, inp, ch in zip(shapes, inputs, caps_host)]
        for t, s, so, ch in zip(tickets, shapes, solo, caps_host):
            check(srv, t, s, so, ch)


def test_start_gate_timeout_fails_alone():
    """The injected request is posted with its start gate shut: the loop's
    bounded wait for it runs out after 20 ms and the request fails with
    -cudaErrorLaunchTimeout; the requests before and after it are exact."""
    shape = (11, 2, 24, 3, 0)
    inputs = [to_dev(O.field_data(4500 + i, shape[2] << shape[0])) for i in range(3)]
    solo = [alone(*shape, inp) for inp in inputs]
    caps_host = [torch.zeros((1 << shape[3]) * 4, dtype=torch.int64).pin_memory() for _ in range(3)]
    with zk.Server(0, 1 << 30, 4, device_loop=True) as srv:
        t0 = srv.submit(*shape, inputs[0], caps_host=caps_host[0])
        check(srv, t0, shape, solo[0], caps_host[0])
        srv.inject_failure(zk.SERVE_FAIL_GATE)
        t1 = srv.submit(*shape, inputs[1], caps_host=caps_host[1])
        r = srv.wait(t1)
        assert r.status == -702, r.status  # -cudaErrorLaunchTimeout
        srv.release(t1)
        t2 = srv.submit(*shape, inputs[2], caps_host=caps_host[2])
        check(srv, t2, shape, solo[2], caps_host[2])


def test_loop_exits_when_idle_and_restarts():
    shape = (10, 3, 16, 4, 3)
    inputs = [to_dev(O.field_data(4600 + i, shape[2] << shape[0])) for i in range(3)]
    solo = [alone(*shape, inp) for inp in inputs]
    caps_host = [torch.zeros((1 << shape[3]) * 4, dtype=torch.int64).pin_memory() for _ in range(3)]
    with zk.Server(0, 1 << 30, 4, device_loop=True) as srv:
        for inp, so, ch in zip(inputs, solo, caps_host):
            t = srv.submit(*shape, inp, caps_host=ch)
            check(srv, t, shape, so, ch)
            time.sleep(0.1)  # longer than the loop's 20 ms idle limit: it exits
        # a kernel on another stream runs once the loop has exited
        x = torch.ones(1 << 20, device="cuda")
        assert float(x.sum()) == float(1 << 20)


def test_unsupported_requests_rejected_at_submit():
    inp = to_dev(O.field_data(1, 16 << 12))
    with zk.Server(0, 1 << 30, 2, device_loop=True) as srv:
        for args in [(8, 2, 16, 2, 0), (23, 1, 1, 0, 0), (12, 2, 16, 2, 5)]:
            with pytest.raises(zk.ZeknoxError):
                srv.submit(*args, inp)
        with pytest.raises(zk.ZeknoxError):
            srv.submit(8, 2, 16, 2, 0, inp, input_is_values=True)


def test_pageable_input_rejected_unless_readable():
    # the server's kernels read the input in place: pageable host memory is
    # refused at submit on a GPU without pageable-memory access (no fault)
    s = (12, 2, 16, 2, 0)
    pageable = torch.from_numpy(O.field_data(17, 16 << 12).view(np.int64).copy())
    assert not pageable.is_pinned()
    from cuda.bindings import runtime as rt

    err, readable = rt.cudaDeviceGetAttribute(rt.cudaDeviceAttr.cudaDevAttrPageableMemoryAccess, 0)
    assert err == rt.cudaError_t.cudaSuccess
    for loop in (False, True):
        with zk.Server(0, 1 << 30, 2, device_loop=loop) as srv:
            if not readable:
                with pytest.raises(zk.ZeknoxError, match="pageable"):
                    srv.submit(*s, pageable)
                assert srv.stats()["completed"] == 0
            else:
                ch = torch.zeros((1 << s[3]) * 4, dtype=torch.int64).pin_memory()
                check(srv, srv.submit(*s, pageable, caps_host=ch), s, alone(*s, pageable.cuda()), ch)


def _corner_columns(lg, seed):
    P = O.P
    n = 1 << lg
    canon = np.array(O.CANONICAL_CORNERS, dtype=np.uint64)
    pick = canon[np.random.default_rng(seed).integers(0, canon.size, n)]
    cols = [np.zeros(n, np.uint64), np.full(n, P - 1, np.uint64), np.tile(np.array([0, P - 1], np.uint64), n // 2),
            np.tile(np.array([P - 1, 1], np.uint64), n // 2), np.full(n, P - (1 << 32), np.uint64),
            np.full(n, (1 << 32) - 1, np.uint64), pick, pick[::-1].copy()]
    return np.concatenate(cols)


@pytest.mark.parametrize("values", [False, True])
@pytest.mark.parametrize("h", [zk.HASH_POSEIDON, zk.HASH_POSEIDON2, zk.HASH_KECCAK])
def test_corner_columns_through_loop_match_oracle(values, h):
    """Columns of field corner values (0, p-1, alternating, p-2^32, 2^32-1,
    corner draws) through the device loop, bit-exact against the oracle."""
    lg, rate, cap = 10, 2, 3
    x = _corner_columns(lg, 990 + h)
    cols = x.size >> lg
    coeffs = O.batched_ntt(x, lg, cols, inverse=True) if values else x
    rows = O.lde_rows(coeffs, lg, rate, cols)
    d, c = O.merkle(rows, cols, cap, h)
    N = 1 << (lg + rate)
    ch = torch.zeros((1 << cap) * 4, dtype=torch.int64).pin_memory()
    inp = to_dev(x)  # held until the request is done
    with zk.Server(0, 1 << 30, 2, device_loop=True) as srv:
        t = srv.submit(lg, rate, cols, cap, h, inp, caps_host=ch, input_is_values=values)
        r = srv.wait(t)
        assert r.status == 2, r.status
        n_dig, _ = zk.merkle_sizes(N, cap)
        assert np.array_equal(device_words(r.leaves, N * cols), rows)
        assert np.array_equal(device_words(r.digests, n_dig * 4).reshape(-1, 4), d)
        assert np.array_equal(ch.numpy().view(np.uint64).reshape(-1, 4), c)
        srv.release(t)
