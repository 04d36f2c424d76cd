"""zeknox_lde_rows_noalloc: the fused LDE for callers that cannot allocate
device memory (their device memory belongs to another allocator or a fixed
arena, or their thread must not enter the driver's allocator).  Called through
the C ABI, it must give the same rows as zeknox_lde_rows, bit for bit, call
after call, without changing the GPU's free memory once its first call has set
it up.

Kept in its own file, collected last, so a stop-at-first-failure run has
already run every other test if this one fails."""
import numpy as np
import pytest
import torch

import zeknox_b200 as zk
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64).copy()).cuda()


def _pair(lg, rate, cols, seed):
    c = _dev(O.field_data(seed, cols << lg))
    ref = torch.zeros(cols << (lg + rate), dtype=torch.int64, device="cuda")
    zk.lde_rows(0, ref, c, lg, rate, cols)
    out = torch.full_like(ref, -1)
    zk.lde_rows_noalloc(0, out, c, lg, rate, cols)
    torch.cuda.synchronize()
    return ref, out


def test_noalloc_matches_lde_rows_twice():
    # first call: full-size rows (2^18 x 40 columns: three chunks), then a second
    # call of another shape right after it
    ref, out = _pair(15, 3, 40, 61)
    assert torch.equal(ref, out)
    ref, out = _pair(11, 2, 24, 62)
    assert torch.equal(ref, out)


def test_noalloc_shape_and_generator_changes():
    # one shape, then another, then the first again, then the first with
    # another coset generator: every call builds its own coset table, so none
    # reads what the previous call left
    for seed, (lg, rate, cols, gen) in enumerate(((12, 3, 20, 7), (9, 1, 16, 7), (12, 3, 20, 7), (12, 3, 20, 11),
                                                   (12, 2, 17, 11), (12, 3, 20, 7))):
        c = _dev(O.field_data(70 + seed, cols << lg))
        ref = torch.zeros(cols << (lg + rate), dtype=torch.int64, device="cuda")
        zk.lde_rows(0, ref, c, lg, rate, cols, coset_gen=gen)
        out = torch.full_like(ref, -1)
        zk.lde_rows_noalloc(0, out, c, lg, rate, cols, coset_gen=gen)
        torch.cuda.synchronize()
        assert torch.equal(ref, out), (lg, rate, cols, gen)


def test_noalloc_allocates_nothing():
    # Each shape is called once first: that call may load kernels lazily and
    # fills the static tables (kernels only).  The repeated call must leave the
    # GPU's free memory exactly as it was.
    for seed, (lg, rate) in ((64, (14, 3)), (65, (9, 1)), (66, (16, 2))):
        cc = _dev(O.field_data(seed, 32 << lg))
        rr = torch.zeros(32 << (lg + rate), dtype=torch.int64, device="cuda")
        zk.lde_rows_noalloc(0, rr, cc, lg, rate, 32)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        rr.fill_(-1)
        torch.cuda.synchronize()
        zk.lde_rows_noalloc(0, rr, cc, lg, rate, 32)
        torch.cuda.synchronize()
        free2, _ = torch.cuda.mem_get_info()
        assert free2 == free1, "device memory changed during the call"
        assert np.array_equal(rr.cpu().numpy().view(np.uint64), O.lde_rows(O.field_data(seed, 32 << lg), lg, rate, 32))


def test_noalloc_rejects_oversize():
    t = torch.zeros(8, dtype=torch.int64, device="cuda")
    with pytest.raises(zk.ZeknoxError) as e:
        zk.lde_rows_noalloc(0, t, t, 17, 2, 1)
    assert "exceeds the static limit" in str(e.value)
