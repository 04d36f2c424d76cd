"""Fused commit path (zeknox_commit / zeknox_lde_rows / zeknox_commit_batch)
vs the oracle: LDE -> bit-reverse transpose -> Merkle forest, bit-exact."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import to_dev, to_np

pytestmark = pytest.mark.gpu


def alloc_job(lg, rate, cols, cap, h, inp, values=False, gen=7):
    N = 1 << (lg + rate)
    leaves = torch.zeros(N * cols, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, cap)
    dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
    caps = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
    job = zk.commit_job(lg, rate, cols, cap, h, inp, leaves, dig, caps, input_is_values=values, coset_gen=gen)
    return job, (leaves, dig, caps, n_dig)


def expect(coeffs, lg, rate, cols, cap, h, gen=7):
    rows = O.lde_rows(coeffs, lg, rate, cols, coset_gen=gen)
    d, c = O.merkle(rows, cols, cap, h)
    return rows, d, c


@pytest.mark.parametrize("lg,rate,cols,cap,h", [
    (1, 1, 1, 0, 3), (2, 2, 3, 1, 0), (4, 3, 16, 2, 3), (6, 1, 17, 0, 4), (9, 3, 8, 4, 1), (10, 2, 33, 3, 3),
    (12, 1, 5, 12, 0), (13, 3, 20, 4, 3), (14, 2, 64, 16, 3), (15, 3, 24, 4, 3), (8, 2, 12, 2, 2)])
def test_commit_matches_oracle(lg, rate, cols, cap, h):
    c = O.field_data(lg * 100 + cols, cols << lg)
    job, (leaves, dig, caps, n_dig) = alloc_job(lg, rate, cols, cap, h, to_dev(c))
    zk.commit(0, job)
    rows, d, cp = expect(c, lg, rate, cols, cap, h)
    assert np.array_equal(to_np(leaves), rows)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4)[:n_dig], d)


def test_commit_from_values():
    lg, rate, cols, cap, h = 11, 2, 12, 3, 3
    vals = O.field_data(5, cols << lg)
    coeffs = O.batched_ntt(vals, lg, cols, inverse=True)
    job, (leaves, dig, caps, n_dig) = alloc_job(lg, rate, cols, cap, h, to_dev(vals), values=True)
    zk.commit(0, job)
    rows, d, cp = expect(coeffs, lg, rate, cols, cap, h)
    assert np.array_equal(to_np(leaves), rows)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)


@pytest.mark.parametrize("lg,rate,cols", [(3, 1, 1), (8, 3, 16), (12, 2, 40), (16, 1, 3), (17, 3, 2)])
def test_lde_rows(lg, rate, cols):
    c = O.field_data(lg + cols, cols << lg)
    rows = torch.zeros(cols << (lg + rate), dtype=torch.int64, device="cuda")
    zk.lde_rows(0, rows, to_dev(c), lg, rate, cols)
    assert np.array_equal(to_np(rows), O.lde_rows(c, lg, rate, cols))


def test_batch_matches_single_jobs():
    shapes = [(10, 1, 8, 2, 0), (12, 3, 20, 4, 3), (9, 2, 64, 1, 4), (11, 3, 3, 0, 1), (13, 1, 17, 5, 3)]
    jobs, bufs, exps = [], [], []
    for i, (lg, rate, cols, cap, h) in enumerate(shapes):
        c = O.field_data(900 + i, cols << lg)
        inp = to_dev(c)
        j, b = alloc_job(lg, rate, cols, cap, h, inp)
        jobs.append(j)
        bufs.append((inp,) + b)
        exps.append(expect(c, lg, rate, cols, cap, h))
    zk.commit_batch(0, jobs)
    for (inp, leaves, dig, caps, n_dig), (rows, d, cp) in zip(bufs, exps):
        assert np.array_equal(to_np(leaves), rows)
        assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
        assert np.array_equal(to_np(dig).reshape(-1, 4)[:n_dig], d)


def test_full_size_workload_properties():
    """256 columns x 2^15 coefficients, rate 3, Poseidon2, cap height 4 (the
    benchmark workload): leaf rows spot-checked against Horner evaluation at
    g * w_N^rev(r), 8 whole columns against the oracle LDE, and the whole
    forest recomputed by the oracle from the GPU leaves."""
    lg, rate, cols, cap, h = 15, 3, 256, 4, 3
    N = 1 << (lg + rate)
    c = O.field_data(2024, cols << lg)
    job, (leaves, dig, caps, n_dig) = alloc_job(lg, rate, cols, cap, h, to_dev(c))
    zk.commit(0, job)
    rows = to_np(leaves).reshape(N, cols)
    rng = np.random.default_rng(7)
    w = O.omega(lg + rate)
    for _ in range(64):
        r, b = int(rng.integers(N)), int(rng.integers(cols))
        i = int(format(r, "018b")[::-1], 2)
        x = O.mul(7, pow(w, i, O.P))
        assert int(rows[r, b]) == O.eval_poly(c[b << lg:(b + 1) << lg], x)
    pick = [0, 1, 77, 128, 200, 253, 254, 255]
    sub = np.concatenate([c[b << lg:(b + 1) << lg] for b in pick])
    ev = O.batched_lde(sub, lg, rate, len(pick))
    for k, b in enumerate(pick):
        col = ev[k * N:(k + 1) * N]
        rev = np.array([int(format(r, "018b")[::-1], 2) for r in range(0, N, 997)])
        assert np.array_equal(rows[::997, b], col[rev])
    d, cp = O.merkle(to_np(leaves), cols, cap, h)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4)[:n_dig], d)


def test_commit_argument_errors():
    t = torch.zeros(64, dtype=torch.int64, device="cuda")
    job, _ = alloc_job(3, 1, 2, 0, 3, t)
    job.rate_bits = 0
    with pytest.raises(zk.ZeknoxError):
        zk.commit(0, job)
    job.rate_bits = 1
    job.hash_type = 5  # no such hash
    with pytest.raises(zk.ZeknoxError):
        zk.commit(0, job)


def test_batch_graph_replay_reads_current_inputs():
    """The cached graph is replayed on the second call with the same buffers:
    new input data must produce the new commitment."""
    shapes = [(11, 2, 24, 3, 3), (9, 3, 7, 2, 0), (12, 1, 16, 4, 4)]
    jobs, bufs = [], []
    for i, (lg, rate, cols, cap, h) in enumerate(shapes):
        inp = to_dev(O.field_data(300 + i, cols << lg))
        j, b = alloc_job(lg, rate, cols, cap, h, inp)
        jobs.append(j)
        bufs.append((inp,) + b)
    zk.commit_batch(0, jobs)
    for rnd in range(2):
        for i, (lg, rate, cols, cap, h) in enumerate(shapes):
            bufs[i][0].copy_(to_dev(O.field_data(400 + 10 * rnd + i, cols << lg)))
        launches = zk.launch_count()
        zk.commit_batch(0, jobs)  # replay: no new host launches
        assert zk.launch_count() == launches
        for i, (lg, rate, cols, cap, h) in enumerate(shapes):
            rows, d, cp = expect(O.field_data(400 + 10 * rnd + i, cols << lg), lg, rate, cols, cap, h)
            inp, leaves, dig, caps, n_dig = bufs[i]
            assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
            assert np.array_equal(to_np(dig).reshape(-1, 4)[:n_dig], d)


def test_commit_on_caller_stream():
    lg, rate, cols, cap, h = 12, 2, 40, 4, 3
    c = O.field_data(77, cols << lg)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        inp = to_dev(c)
        job, (leaves, dig, caps, n_dig) = alloc_job(lg, rate, cols, cap, h, inp)
        zk.commit(0, job, stream=s.cuda_stream)
    s.synchronize()
    rows, d, cp = expect(c, lg, rate, cols, cap, h)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("lg,rate,cols", [(13, 3, 72), (15, 3, 100), (16, 2, 81)])
def test_commit_from_host_memory(pinned, lg, rate, cols):
    """zeknox_commit with a host input pointer stages the coefficients itself
    (chunked copies overlapping the LDE; the larger shapes take several
    chunks); same commitment as a device input."""
    cap, h = 4, 3
    c = O.field_data(88, cols << lg)
    host = torch.from_numpy(c.view(np.int64).copy())
    if pinned:
        host = host.pin_memory()
    job, (leaves, dig, caps, n_dig) = alloc_job(lg, rate, cols, cap, h, host)
    zk.commit(0, job)
    rows, d, cp = expect(c, lg, rate, cols, cap, h)
    assert np.array_equal(to_np(leaves), rows)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    assert np.array_equal(to_np(dig).reshape(-1, 4)[:n_dig], d)


@pytest.mark.parametrize("lg,rate,cols,n_dst,n_src", [(10, 2, 24, 4, 3), (15, 3, 40, 2, 2), (6, 1, 5, 1, 2),
                                                      (12, 3, 17, 8, 4)])
def test_lde_rows_scatter_assembles_row_shards(lg, rate, cols, n_dst, n_src):
    """Several column shards (the sources of a multi-GPU commit) each scatter
    their LDE rows into n_dst row-shard buffers (the destinations, emulated as
    buffers of this GPU); every destination must end up holding its block of
    whole leaf rows, exactly the single-call LDE's."""
    n, N = 1 << lg, 1 << (lg + rate)
    c = O.field_data(lg * 3 + cols, cols * n)
    rows = O.lde_rows(c, lg, rate, cols).reshape(N, cols)
    per = N // n_dst
    dst = [torch.zeros(per * cols, dtype=torch.int64, device="cuda") for _ in range(n_dst)]
    base, rem = divmod(cols, n_src)
    c0 = 0
    for s in range(n_src):
        k = base + (1 if s < rem else 0)
        if k:
            zk.lde_rows_scatter(0, dst, to_dev(c[c0 * n:(c0 + k) * n]), lg, rate, k, c0, cols)
        c0 += k
    for d in range(n_dst):
        assert np.array_equal(to_np(dst[d]).reshape(per, cols), rows[d * per:(d + 1) * per])


def test_lde_rows_scatter_argument_errors():
    t = torch.zeros(64, dtype=torch.int64, device="cuda")
    with pytest.raises(zk.ZeknoxError):
        zk.lde_rows_scatter(0, [t, t, t], t, 3, 1, 1, 0, 1)  # 3 destinations: not a power of two
    with pytest.raises(zk.ZeknoxError):
        zk.lde_rows_scatter(0, [t, t], t, 3, 1, 2, 1, 2)  # columns beyond the rows
