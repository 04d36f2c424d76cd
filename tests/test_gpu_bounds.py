"""The range-checked build (libzeknox_checked.so: every global index of the
NTT, reorder, transpose and Merkle kernels tested against its buffer's extent;
an access out of range is skipped and recorded, never made) runs the parity
shapes -- ragged and small sizes, every hash, the fused LDE and commit, the
host-input and multi-chunk paths -- in a fresh process, and must record no
out-of-range access while still matching the oracle bit for bit.  The GPU has
no sanitizer here; this and the canary tests stand in for it."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "zeknox_b200", "libzeknox_checked.so")

SCRIPT = r'''
import sys
import numpy as np
import torch
sys.path.insert(0, ROOT)
import zeknox_b200 as zk
from oracle import oracle as O
from tests.helpers import HASHES, to_dev, to_np

checked, rec = zk.bounds_report(0)
assert checked, "not the checked build: " + zk.LIB_PATH
n_cases = 0

def clean(what):
    global n_cases
    ok, r = zk.bounds_report(0)
    assert r[0] == 0, "%s: %d out-of-range accesses, first at site %d index %d extent %d" % (what, *r)
    n_cases += 1

for lg, b in [(1, 1), (4, 3), (9, 5), (12, 7), (16, 2), (18, 1)]:
    x = O.field_data(lg + b, b << lg)
    for inv, coset in [(False, False), (True, False), (False, True), (True, True)]:
        t = to_dev(x)
        zk.ntt_batch(0, t, lg, b, with_coset=coset, inverse=inv)
        assert np.array_equal(to_np(t), O.batched_ntt(x, lg, b, inverse=inv, with_coset=coset))
        clean("ntt %d %d" % (lg, b))
for lg, rate, b in [(1, 1, 1), (5, 3, 3), (10, 2, 17), (13, 3, 20), (15, 3, 40), (17, 1, 3)]:
    c = O.field_data(7 * lg + b, b << lg)
    out = torch.zeros(b << (lg + rate), dtype=torch.int64, device="cuda")
    zk.lde_batch(0, out, to_dev(c), lg, b, rate)
    assert np.array_equal(to_np(out), O.batched_lde(c, lg, rate, b))
    clean("lde")
    rows = torch.zeros_like(out)
    zk.lde_rows(0, rows, to_dev(c), lg, rate, b)
    assert np.array_equal(to_np(rows), O.lde_rows(c, lg, rate, b))
    clean("lde_rows")
    if lg >= 10:
        out2 = torch.zeros(b << (lg + rate), dtype=torch.int64)
        zk.lde_batch(0, out2, torch.from_numpy(c.view(np.int64).copy()), lg, b, rate)
        assert np.array_equal(out2.numpy().view(np.uint64), O.batched_lde(c, lg, rate, b))
        clean("lde host buffers")
for lg, b in [(0, 3), (3, 5), (7, 33), (10, 64), (12, 6)]:
    x = O.field_data(lg * 3 + b, b << lg)
    out = torch.zeros(b << lg, dtype=torch.int64, device="cuda")
    zk.transpose_rev_batch(0, out, to_dev(x), lg, b)
    assert np.array_equal(to_np(out), O.transpose_rev(x, lg, b))
    clean("transpose")
for name, h in HASHES.items():
    for nl, ls, ch in [(1 << 9, 9, 2), (1 << 8, 3, 1), (1 << 6, 135, 6), (1 << 12, 17, 0), (1 << 14, 8, 4),
                       (1 << 11, 4, 3)]:
        if h == zk.HASH_POSEIDON_BN128 and nl * ls > (1 << 16):
            continue
        leaves = O.field_data(nl + ls + h, nl * ls)
        n_dig, n_cap = zk.merkle_sizes(nl, ch)
        dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
        cap = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
        zk.fill_digests_buf_linear_gpu(dig, cap, to_dev(leaves), nl, ls, ch, h)
        d, cp = O.merkle(leaves, ls, ch, h)
        assert np.array_equal(to_np(cap).reshape(-1, 4), cp), (name, nl, ls, ch)
        if n_dig:
            assert np.array_equal(to_np(dig).reshape(-1, 4)[:n_dig], d), (name, nl, ls, ch)
        clean("forest %s %d %d %d" % (name, nl, ls, ch))
for lg, rate, cols, cap, h in [(3, 1, 5, 1, 3), (9, 3, 19, 4, 0), (8, 2, 1, 10, 1), (14, 2, 64, 4, 3),
                               (12, 3, 24, 4, 4)]:
    c = O.field_data(lg * 31 + cols, cols << lg)
    N = 1 << (lg + rate)
    n_dig, n_cap = zk.merkle_sizes(N, cap)
    leaves = torch.zeros(N * cols, dtype=torch.int64, device="cuda")
    dig = torch.zeros(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
    caps = torch.zeros(n_cap * 4, dtype=torch.int64, device="cuda")
    zk.commit(0, zk.commit_job(lg, rate, cols, cap, h, to_dev(c), leaves, dig, caps))
    rows = O.lde_rows(c, lg, rate, cols)
    d, cp = O.merkle(rows, cols, cap, h)
    assert np.array_equal(to_np(leaves), rows)
    assert np.array_equal(to_np(caps).reshape(-1, 4), cp)
    clean("commit")
print("bounds clean over %d cases" % n_cases)
'''


@pytest.mark.skipif(not os.path.exists(CHECKED), reason="checked build not made (make -C zeknox_b200 checked)")
def test_checked_build_records_no_out_of_range_access():
    env = dict(os.environ, ZEKNOX_LIB=CHECKED, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + SCRIPT], env=env, capture_output=True,
                       text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "bounds clean" in r.stdout


def test_normal_build_reports_no_checks():
    import zeknox_b200 as zk
    checked, rec = zk.bounds_report(0)
    assert not checked and rec == [0, 0, 0, 0]
