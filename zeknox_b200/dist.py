"""One commit spread over the ranks of a process group (one process per GPU).

The commit has exactly one exchange step (LDE columns are independent; Merkle
subtrees need whole leaf rows):

1. every rank extends its shard of the columns (``multi.split_columns``) into
   bit-reversed leaf rows of its own columns, on its GPU;
2. one ``all_to_all_single`` moves row block d (the rows of the subtrees
   hashed by rank d, ``multi.split_subtrees``) of every rank's columns to
   rank d -- over NVLink with NCCL, or through gloo on CPU;
3. each hashing rank interleaves the column blocks it received into whole
   leaf rows and builds the forest of its subtrees; its digests are the
   sub-range of the single-GPU digest buffer that belongs to those subtrees;
4. one ``all_gather`` hands every rank all caps.

Exchange volume per rank: N * cols * 8 * (G - 1) / G bytes for G hashing
ranks.

``commit_distributed_p2p`` fuses steps 1 and 2: every hashing rank exports its
row shard with a CUDA IPC handle, every other rank maps it, and each rank's
row-writing LDE kernel stores its columns of every row straight into the
owning rank's shard (``zeknox_lde_rows_scatter``: plain P2P stores over
NVLink, no staging buffer, no separate collective), so the exchange overlaps
the transform tile by tile.  The shards are ordinary device allocations: no
NVLink multicast object is created or bound.

zeknox itself has no multi-process commit: its multi-GPU entry points
(native/ntt/ntt.cu:315-471, native/merkle/merkle.cu:283-499) drive several GPUs
from one process and partition the same way (columns for the LDE, whole
subtrees for the Merkle forest); this module is that partitioning with the
row exchange the two partitions imply.

The compute steps are callables so that the exchange and assembly logic can
be exercised on CPU ranks (gloo) with any implementation of the two stages;
``commit_distributed`` uses this library's CUDA kernels.
"""
import torch
import torch.distributed as dist

from .multi import merkle_gpus, split_columns


def _log2(x):
    assert x > 0 and x & (x - 1) == 0, x
    return x.bit_length() - 1


def commit_sharded(coeffs, lg_n, rate_bits, cols, cap_height, lde, merkle, group=None):
    """Generic form of the distributed commit.

    coeffs: this rank's columns, a flat tensor of k * 2^lg_n coefficients
      (column-major; k and the first column from ``split_columns(cols, world)``).
    lde(coeffs, k) -> flat tensor of 2^(lg_n + rate_bits) * k words: the
      bit-reversed leaf rows of this rank's k columns (row-major, k wide).
    merkle(leaves, n_leaves, leaf_size, cap_height) -> (digests, caps) flat
      tensors (digests may be empty when the subtrees are single leaves).

    Returns (caps, digests, leaves): caps of the whole forest (every rank,
    n_caps * 4 words), and on a hashing rank the digests of its subtrees and
    its leaf rows (None elsewhere)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    N = 1 << (lg_n + rate_bits)
    n_caps = 1 << cap_height
    shards = split_columns(cols, world)
    _, k = shards[rank]
    G = merkle_gpus(n_caps, world)
    rows_per = N // G
    if k:
        rows = lde(coeffs, k)
        assert rows.numel() == N * k
    else:
        rows = torch.empty(0, dtype=torch.int64, device=coeffs.device)
    # rows [d * rows_per, (d + 1) * rows_per) of my columns go to rank d < G
    in_split = [rows_per * k if d < G else 0 for d in range(world)]
    out_split = [rows_per * k_s if rank < G else 0 for _, k_s in shards]
    recv = torch.empty(sum(out_split), dtype=rows.dtype, device=rows.device)
    dist.all_to_all_single(recv, rows.contiguous(), output_split_sizes=out_split, input_split_sizes=in_split,
                           group=group)
    caps_g = n_caps // G
    digests = leaves = None
    if rank < G:
        leaves = torch.empty(rows_per * cols, dtype=recv.dtype, device=recv.device)
        lv = leaves.view(rows_per, cols)
        off = 0
        for c_s, k_s in shards:
            if k_s:
                lv[:, c_s:c_s + k_s] = recv[off:off + rows_per * k_s].view(rows_per, k_s)
                off += rows_per * k_s
        digests, my_caps = merkle(leaves, rows_per, cols, _log2(caps_g))
    else:
        my_caps = torch.zeros(caps_g * 4, dtype=recv.dtype, device=recv.device)
    gathered = [torch.empty(caps_g * 4, dtype=recv.dtype, device=recv.device) for _ in range(world)]
    dist.all_gather(gathered, my_caps.contiguous(), group=group)
    caps = torch.cat(gathered[:G])
    return caps, digests, leaves


def commit_distributed(coeffs, lg_n, rate_bits, cols, cap_height, hash_type, coset_gen=7, group=None, device_id=None,
                       stream=None):
    """The distributed commit on this rank's GPU (NCCL process group): the LDE
    is ``zeknox_lde_rows`` of the local columns, the forest
    ``fill_digests_buf_linear_gpu_with_gpu_ptr`` of the local subtrees.
    coeffs: CUDA int64 tensor of this rank's columns (see commit_sharded)."""
    from . import fill_digests_buf_linear_gpu, lde_rows, merkle_sizes

    if not coeffs.is_cuda:
        raise ValueError("commit_distributed takes CUDA tensors (use commit_sharded for other stages)")
    dev = coeffs.device.index if device_id is None else device_id
    N = 1 << (lg_n + rate_bits)

    def lde(c, k):
        rows = torch.empty(N * k, dtype=torch.int64, device=c.device)
        lde_rows(dev, rows, c, lg_n, rate_bits, k, coset_gen, stream=stream)
        return rows

    def merkle(leaves, n_leaves, leaf_size, h):
        n_dig, n_cap = merkle_sizes(n_leaves, h)
        dig = torch.empty(max(n_dig, 1) * 4, dtype=torch.int64, device=leaves.device)
        caps = torch.empty(n_cap * 4, dtype=torch.int64, device=leaves.device)
        torch.cuda.synchronize(leaves.device)  # the Merkle entry point queues on the legacy default stream
        fill_digests_buf_linear_gpu(dig, caps, leaves, n_leaves, leaf_size, h, hash_type, gpu_id=dev)
        torch.cuda.synchronize(leaves.device)
        return dig[:n_dig * 4], caps

    return commit_sharded(coeffs, lg_n, rate_bits, cols, cap_height, lde, merkle, group=group)


def _mapped_shards(buf, G, group):
    """Device addresses, in this process, of the G hashing ranks' row shards.
    Each owner exports its shard (``buf`` on ranks < G) as a CUDA IPC handle
    (cudaIpcGetMemHandle, through torch's CUDA tensor sharing); every rank
    maps the others' shards (cudaIpcOpenMemHandle).  Returns the addresses and
    the mapped tensors, which must stay alive while the addresses are used."""
    from torch.multiprocessing.reductions import reduce_tensor

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    handles = [None] * world
    dist.all_gather_object(handles, reduce_tensor(buf) if rank < G else None, group=group)
    ptrs, keep = [], []
    for r in range(G):
        if r == rank:
            ptrs.append(buf.data_ptr())
        else:
            rebuild, args = handles[r]
            t = rebuild(*args)
            keep.append(t)
            ptrs.append(t.data_ptr())
    return ptrs, keep


def commit_distributed_p2p(coeffs, lg_n, rate_bits, cols, cap_height, hash_type, coset_gen=7, group=None,
                           device_id=None):
    """The distributed commit with the row exchange fused into the LDE: the
    hashing ranks' row shards are mapped into every rank's address space by
    CUDA IPC handles, every rank's ``zeknox_lde_rows_scatter`` writes its
    columns of each row directly into the owner's shard, then a host barrier
    and the local forests as in ``commit_distributed``.  Same arguments and
    results."""
    from . import fill_digests_buf_linear_gpu, lde_rows_scatter, merkle_sizes

    if not coeffs.is_cuda:
        raise ValueError("commit_distributed_p2p takes CUDA tensors")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = coeffs.device.index if device_id is None else device_id
    N = 1 << (lg_n + rate_bits)
    n_caps = 1 << cap_height
    shards = split_columns(cols, world)
    c0, k = shards[rank]
    G = merkle_gpus(n_caps, world)
    rows_per = N // G
    buf = torch.empty(rows_per * cols if rank < G else 0, dtype=torch.int64, device=coeffs.device)
    ptrs, mapped = _mapped_shards(buf, G, group)
    if k:
        lde_rows_scatter(dev, ptrs, coeffs, lg_n, rate_bits, k, c0, cols, coset_gen)  # waits for its kernels
    torch.cuda.synchronize(coeffs.device)
    dist.barrier(group=group)  # every rank's stores have landed before any forest starts
    caps_g = n_caps // G
    digests = leaves = None
    if rank < G:
        leaves = buf
        h = _log2(caps_g)
        n_dig, n_cap = merkle_sizes(rows_per, h)
        dig = torch.empty(max(n_dig, 1) * 4, dtype=torch.int64, device=coeffs.device)
        my_caps = torch.empty(n_cap * 4, dtype=torch.int64, device=coeffs.device)
        fill_digests_buf_linear_gpu(dig, my_caps, leaves, rows_per, cols, h, hash_type, gpu_id=dev)
        torch.cuda.synchronize(coeffs.device)
        digests = dig[:n_dig * 4]
    else:
        my_caps = torch.zeros(caps_g * 4, dtype=torch.int64, device=coeffs.device)
    gathered = [torch.empty(caps_g * 4, dtype=torch.int64, device=coeffs.device) for _ in range(world)]
    dist.all_gather(gathered, my_caps, group=group)
    # no rank may reuse or free its shard while another rank could still be
    # writing it or still holds its mapping
    del mapped
    dist.barrier(group=group)
    return torch.cat(gathered[:G]), digests, leaves
