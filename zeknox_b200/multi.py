"""Multi-GPU partitioning of the commit path (host logic).

The path shards by independent objects, with no exchange inside a commit:
  * LDE columns: the first (batches % G) GPUs take one column more, as
    zeknox's batch_lde_multi_gpu (native/ntt/ntt.cu:324-337) and this
    library's compute_batched_lde_multi_gpu do;
  * Merkle subtrees: a power-of-two number of GPUs G' <= min(G, caps) each
    builds caps / G' whole subtrees (fill_digests_buf_linear_multigpu_with_gpu_ptr);
    a subtree's digests and cap are contiguous in the linear layout, so shard
    g's outputs are plain sub-ranges of the full buffers.
These functions give the exact ranges the C++ entry points use; the tests run
them across gloo ranks on CPU and check that the shards assemble into the
single-process result.
"""


def split_columns(batches, world):
    """[(first_column, count)] per rank."""
    base, rem = divmod(batches, world)
    out, first = [], 0
    for g in range(world):
        take = base + (1 if g < rem else 0)
        out.append((first, take))
        first += take
    return out


def merkle_gpus(n_caps, world):
    """Number of GPUs the Merkle forest is split over: the largest power of two
    <= world that divides the caps."""
    g = 1
    while g * 2 <= world and g * 2 <= n_caps:
        g *= 2
    return g


def split_subtrees(n_leaves, n_caps, world):
    """Per used rank: dict with the leaf, digest and cap ranges (in leaves,
    digests and caps) of its whole subtrees, plus its sub-forest cap height."""
    G = merkle_gpus(n_caps, world)
    L = n_leaves // n_caps
    D = 2 * L - 2
    caps_g = n_caps // G
    h = caps_g.bit_length() - 1
    shards = []
    for g in range(G):
        shards.append({"rank": g, "leaves": (g * caps_g * L, caps_g * L), "digests": (g * caps_g * D, caps_g * D),
                       "caps": (g * caps_g, caps_g), "cap_height": h})
    return shards
