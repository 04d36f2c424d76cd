"""Multi-GPU partitioning checked across 2 gloo ranks on CPU.

Each rank builds only its shard -- its LDE columns (oracle LDE) and its Merkle
subtrees (the library's exported CPU builder, fill_digests_buf_linear_cpu) --
the shards are all-gathered, and rank 0 checks that they assemble into exactly
the single-process commitment."""
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


def _worker(rank, world, port, result):
    import zeknox_b200 as zk
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # ---- LDE columns
        lg, rate, cols = 7, 2, 11
        n, N = 1 << lg, 1 << (lg + rate)
        coeffs = O.field_data(123, cols * n)
        first, take = multi.split_columns(cols, world)[rank]
        mine = O.batched_lde(coeffs[first * n:(first + take) * n], lg, rate, take) if take else np.zeros(0, np.uint64)
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        lde_ok = np.array_equal(np.concatenate(parts), O.batched_lde(coeffs, lg, rate, cols))
        # ---- Merkle subtrees
        n_leaves, leaf_size, cap_h, h = 256, 13, 3, 3
        leaves = O.field_data(77, n_leaves * leaf_size)
        shards = multi.split_subtrees(n_leaves, 1 << cap_h, world)
        out = None
        for sh in shards:
            if sh["rank"] != rank:
                continue
            l0, ln = sh["leaves"]
            lv = torch.from_numpy(leaves[l0 * leaf_size:(l0 + ln) * leaf_size].view(np.int64).copy())
            nd, nc = zk.merkle_sizes(ln, sh["cap_height"])
            dg = torch.zeros(max(nd, 1) * 4, dtype=torch.int64)
            cp = torch.zeros(nc * 4, dtype=torch.int64)
            zk.fill_digests_buf_linear_cpu(dg, cp, lv, ln, leaf_size, sh["cap_height"], h)
            out = (dg.numpy().view(np.uint64)[:nd * 4].copy(), cp.numpy().view(np.uint64).copy())
        got = [None] * world
        dist.all_gather_object(got, out)
        d_full, c_full = O.merkle(leaves, leaf_size, cap_h, h)
        dig = np.concatenate([g[0] for g in got if g is not None]).reshape(-1, 4)
        cap = np.concatenate([g[1] for g in got if g is not None]).reshape(-1, 4)
        merkle_ok = np.array_equal(dig, d_full) and np.array_equal(cap, c_full)
        if rank == 0:
            result.put((bool(lde_ok), bool(merkle_ok)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_shards_assemble_into_single_process_result(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    lde_ok, merkle_ok = q.get(timeout=5)
    assert lde_ok and merkle_ok



def test_partition_rules():
    assert multi.split_columns(10, 4) == [(0, 3), (3, 3), (6, 2), (8, 2)]
    assert multi.merkle_gpus(16, 8) == 8 and multi.merkle_gpus(16, 6) == 4 and multi.merkle_gpus(2, 8) == 2
    sh = multi.split_subtrees(64, 8, 4)
    assert [s["caps"] for s in sh] == [(0, 2), (2, 2), (4, 2), (6, 2)]
    assert sh[1]["digests"] == (2 * 14, 2 * 14) and sh[1]["cap_height"] == 1


def test_cxx_partition_matches_host_partition(tmp_path):
    """The C++ partition the multi-GPU entry points use (multi_split.h), compiled
    on its own, gives the same column runs and subtree GPU counts as the host
    functions the process-group path uses, for 1..8 GPUs."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "split.cpp"
    src.write_text('#include <stdio.h>\n#include "multi_split.h"\n'
                   'int main(){for(unsigned g=1;g<=8;g++)for(unsigned b=0;b<=40;b++){'
                   'zk::ColumnSplit s=zk::split_columns(b,g);'
                   'for(unsigned k=0;k<g;k++)printf("%u %u %u %llu %llu\\n",g,b,k,'
                   '(unsigned long long)s.first[k],(unsigned long long)s.take[k]);}'
                   'for(unsigned g=1;g<=8;g++)for(unsigned c=1;c<=256;c*=2)'
                   'printf("m %u %u %llu\\n",g,c,(unsigned long long)zk::merkle_gpu_count(g,c));return 0;}\n')
    exe = tmp_path / "split"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(root, "zeknox_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    n_cols = n_merkle = 0
    for line in lines:
        f = line.split()
        if f[0] == "m":
            g, c, count = map(int, f[1:])
            assert count == multi.merkle_gpus(c, g), line
            n_merkle += 1
        else:
            g, b, k, first, take = map(int, f)
            assert (first, take) == multi.split_columns(b, g)[k], line
            n_cols += 1
    assert n_cols == sum(g * 41 for g in range(1, 9)) and n_merkle == 8 * 9
