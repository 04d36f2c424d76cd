"""GPU NTT / LDE / transpose through the C ABI vs the oracle; bit-exact."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import to_dev, to_np

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 4, 5, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 20]


@pytest.mark.parametrize("lg", SIZES)
@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("coset", [False, True])
def test_ntt_device(lg, inverse, coset):
    batches = 3 if lg <= 16 else 1
    x = O.field_data(lg * 7 + inverse, batches << lg)
    t = to_dev(x)
    zk.ntt_batch(0, t, lg, batches, with_coset=coset, inverse=inverse)
    exp = O.batched_ntt(x, lg, batches, inverse=inverse, with_coset=coset)
    assert np.array_equal(to_np(t), exp)


@pytest.mark.parametrize("lg", [4, 12, 17])
def test_ntt_host_buffers(lg):
    x = O.field_data(lg, 2 << lg)
    t = torch.from_numpy(x.view(np.int64).copy())
    zk.ntt_batch(0, t, lg, 2)
    assert np.array_equal(t.numpy().view(np.uint64), O.batched_ntt(x, lg, 2))
    zk.intt_batch(0, t, lg, 2)
    assert np.array_equal(t.numpy().view(np.uint64), x)


@pytest.mark.parametrize("lg,rate,batches", [(1, 1, 2), (2, 3, 5), (4, 1, 2), (9, 3, 3), (10, 2, 7), (12, 1, 2),
                                             (13, 3, 4), (15, 3, 2), (17, 3, 1), (18, 1, 2)])
@pytest.mark.parametrize("coset", [True, False])
def test_lde_device(lg, rate, batches, coset):
    c = O.field_data(lg * 13 + rate, batches << lg)
    out = torch.zeros(batches << (lg + rate), dtype=torch.int64, device="cuda")
    zk.lde_batch(0, out, to_dev(c), lg, batches, rate, with_coset=coset)
    assert np.array_equal(to_np(out), O.batched_lde(c, lg, rate, batches, with_coset=coset))


@pytest.mark.parametrize("lg,rate", [(3, 1), (10, 2), (14, 1)])
def test_lde_inverse_direction(lg, rate):
    c = O.field_data(lg, 2 << lg)
    out = torch.zeros(2 << (lg + rate), dtype=torch.int64, device="cuda")
    zk.lde_batch(0, out, to_dev(c), lg, 2, rate, with_coset=True, inverse=True)
    assert np.array_equal(to_np(out), O.batched_lde(c, lg, rate, 2, inverse=True, with_coset=True))


def test_lde_host_buffers_and_salt():
    lg, rate, b, salt = 11, 2, 3, 2
    c = O.field_data(5, b << lg)
    out = torch.zeros((b + salt) << (lg + rate), dtype=torch.int64)
    zk.lde_batch(0, out, torch.from_numpy(c.view(np.int64).copy()), lg, b, rate, salt_size=salt)
    got = out.numpy().view(np.uint64)
    N = 1 << (lg + rate)
    assert np.array_equal(got[:b * N], O.batched_lde(c, lg, rate, b))
    s = got[b * N:]
    assert (s < np.uint64(O.P)).all() and len(np.unique(s)) > 0.99 * s.size


def test_custom_coset_generator():
    lg, rate = 8, 2
    zk.init_coset(0, lg + rate, 11)
    try:
        c = O.field_data(9, 2 << lg)
        out = torch.zeros(2 << (lg + rate), dtype=torch.int64, device="cuda")
        zk.lde_batch(0, out, to_dev(c), lg, 2, rate, with_coset=True)
        assert np.array_equal(to_np(out), O.batched_lde(c, lg, rate, 2, coset_gen=11))
        t = to_dev(c)
        zk.ntt_batch(0, t, lg, 2, with_coset=True)
        assert np.array_equal(to_np(t), O.batched_ntt(c, lg, 2, with_coset=True, coset_gen=11))
    finally:
        zk.init_coset(0, 20, 7)


@pytest.mark.parametrize("lg,b", [(0, 3), (1, 1), (1, 2), (5, 3), (6, 30), (6, 31), (10, 33), (12, 256), (17, 7),
                                  (20, 2)])
def test_transpose_rev(lg, b):
    x = O.field_data(lg + b, b << lg)
    out = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
    zk.transpose_rev_batch(0, out, to_dev(x), lg, b)
    assert np.array_equal(to_np(out), O.transpose_rev(x, lg, b))
    out2 = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
    zk.transpose_rev_batch(0, out2, to_dev(x), lg, b, naive=True)
    assert torch.equal(out, out2)
    # the stream-ordered extension entry point
    s = torch.cuda.Stream()
    out3 = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
    src = to_dev(x)
    torch.cuda.synchronize()
    zk.transpose_rev(0, out3, src, lg, b, stream=s.cuda_stream)
    s.synchronize()
    assert torch.equal(out, out3)


@pytest.mark.parametrize("lg,b", [(9, 64), (12, 6)])
def test_transpose_rev_unaligned_buffers(lg, b):
    """Buffers that start 8 bytes past a 16-byte boundary take the 8-byte
    form; both forms give the oracle's matrix."""
    x = O.field_data(77 + lg, b << lg)
    src = torch.zeros((b << lg) + 1, dtype=torch.int64, device="cuda")
    src[1:] = to_dev(x)
    out = torch.zeros((b << lg) + 1, dtype=torch.int64, device="cuda")
    zk.transpose_rev_batch(0, out[1:], src[1:], lg, b)
    assert np.array_equal(to_np(out[1:]), O.transpose_rev(x, lg, b))
    aligned = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
    zk.transpose_rev_batch(0, aligned, src[1:], lg, b)
    assert torch.equal(aligned, out[1:])


@pytest.mark.parametrize("lg,b", [(6, 2), (6, 64), (7, 34), (11, 96), (13, 258), (16, 40), (18, 64)])
def test_transpose_rev_bulk_and_plain_forms(lg, b):
    """Every tile shape of the bulk-copy staged transpose (knob
    transpose_bulk 1..8: persistent CTAs, 2-8 stages; ragged last column tile,
    fewer tiles than CTAs, many tiles per CTA) and the 16-byte form (0) give
    the oracle's matrix."""
    x = O.field_data(5 * lg + b, b << lg)
    src = to_dev(x)
    exp = O.transpose_rev(x, lg, b)
    outs = []
    try:
        for form in (1, 2, 3, 4, 5, 6, 7, 8, 0):
            zk.tune_set("transpose_bulk", form)
            out = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
            zk.transpose_rev_batch(0, out, src, lg, b)
            outs.append(out)
    finally:
        zk.tune_set("transpose_bulk", zk.TRANSPOSE_AUTO)
    assert np.array_equal(to_np(outs[0]), exp)
    for o in outs[1:]:
        assert torch.equal(outs[0], o)


def test_transpose_rev_bounded_wait_times_out():
    """A stage whose byte count never completes (injected: 16 bytes declared
    and not copied) ends its CTA's wait after the limit; the call returns
    -cudaErrorLaunchTimeout, and the next transposes on the same context are
    bit-exact.  Nothing faults or hangs: the copies all complete, only the
    barrier's expected count is never reached."""
    lg, b = 12, 64
    x = O.field_data(4242, b << lg)
    src = to_dev(x)
    out = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
    zk.inject_wait_timeout(0, 1)
    with pytest.raises(zk.ZeknoxError) as e:
        zk.transpose_rev_batch(0, out, src, lg, b)
    assert e.value.code == -702  # cudaErrorLaunchTimeout
    for _ in range(2):
        out = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
        zk.transpose_rev_batch(0, out, src, lg, b)
        assert np.array_equal(to_np(out), O.transpose_rev(x, lg, b))


def test_argument_errors():
    t = torch.zeros(16, dtype=torch.int64, device="cuda")
    with pytest.raises(zk.ZeknoxError) as e:
        zk.ntt_batch(0, t, 0, 1)
    assert e.value.code == 1
    with pytest.raises(zk.ZeknoxError) as e:
        zk.lde_batch(0, t, t, 2, 1, 0)
    assert e.value.code == 1
    with pytest.raises(zk.ZeknoxError):
        zk.ntt_batch(99, t, 2, 1)


def test_init_entry_points():
    assert zk.cuda_available()
    assert zk.get_number_of_gpus() >= 1
    zk.init_twiddle_factors(0, 16)
    zk.init_cuda_degree(20)


def test_lde_multi_gpu_entry_matches_single():
    """compute_batched_lde_multi_gpu on the GPUs present (one on this test's
    machine) against compute_batched_lde, batches 1..9 at lg 17, rate 3, as the
    reference's wrappers/rust/tests/ntt.rs:578-661 does: host input, output in
    GPU 0's memory."""
    lg, rate = 17, 3
    ngpu = zk.get_number_of_gpus()
    host = O.field_data(171, 9 << lg)
    out = torch.zeros(9 << (lg + rate), dtype=torch.int64, device="cuda")
    for batches in range(1, 10):
        inp = torch.from_numpy(host[:batches << lg].view(np.int64).copy())
        out.fill_(-1)
        zk.lde_batch_multi_gpu(out, inp, ngpu, lg, batches, rate)
        single = torch.zeros(batches << (lg + rate), dtype=torch.int64)
        zk.lde_batch(0, single, inp, lg, batches, rate)
        assert torch.equal(out[:batches << (lg + rate)].cpu(), single), batches
    # and against the oracle on the last, largest call
    assert np.array_equal(single.numpy().view(np.uint64), O.batched_lde(host, lg, rate, 9))
