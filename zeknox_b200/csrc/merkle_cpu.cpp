// merkle_cpu.cpp -- fill_digests_buf_linear_cpu, the library's host Merkle builder.
//
// The reference exports a CPU twin of the GPU builder
// (native/merkle/merkle.cpp:126-161); this is the same contract implemented on
// this library's host-compiled hashers (hash.cuh) with OpenMP over leaves and
// over the nodes of each level.
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "geom.h"
#include "hash.cuh"

template <int H>
static void build(uint64_t *dig, uint64_t *cap, const uint64_t *leaves, uint64_t n_dig, uint64_t n_cap, uint64_t n_leaves,
                  uint64_t leaf_size, uint64_t cap_height)
{
    if (n_cap == n_leaves) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n_leaves; i++) zk::hash_one<H>(leaves + i * leaf_size, leaf_size, cap + 4 * i);
        return;
    }
    const uint64_t L = n_leaves >> cap_height, D = n_dig >> cap_height;
    for (uint64_t k = 0; k < n_cap; k++) {
        const uint64_t *lv = leaves + k * L * leaf_size;
        uint64_t *dg = dig + k * D * 4;
        uint64_t *cp = cap + k * 4;
        uint64_t *leaf_dig = dg + (D - L) * 4;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)L; i++) zk::hash_one<H>(lv + i * leaf_size, leaf_size, leaf_dig + 4 * i);
        for (uint64_t level = L / 2; level >= 2; level /= 2) {
            const uint64_t start = level - 2, child = 2 * level - 2;
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < (int64_t)level; i++)
                zk::hash_two<H>(dg + 4 * (child + 2 * i), dg + 4 * (child + 2 * i + 1), dg + 4 * (start + i));
        }
        zk::hash_two<H>(dg, dg + 4, cp);
    }
}

bool zk_merkle_cpu(void *digests, void *caps, const void *leaves, uint64_t n_dig, uint64_t n_cap, uint64_t n_leaves,
                   uint64_t leaf_size, uint64_t cap_height, uint64_t hash_type, std::string &err)
{
    if (!zk::merkle_geometry_check(n_dig, n_cap, n_leaves, cap_height, err)) return false;
    uint64_t *d = (uint64_t *)digests, *c = (uint64_t *)caps;
    const uint64_t *l = (const uint64_t *)leaves;
    switch (hash_type) {
    case zk::HASH_POSEIDON: build<zk::HASH_POSEIDON>(d, c, l, n_dig, n_cap, n_leaves, leaf_size, cap_height); break;
    case zk::HASH_KECCAK: build<zk::HASH_KECCAK>(d, c, l, n_dig, n_cap, n_leaves, leaf_size, cap_height); break;
    case zk::HASH_POSEIDON_BN128:
        build<zk::HASH_POSEIDON_BN128>(d, c, l, n_dig, n_cap, n_leaves, leaf_size, cap_height);
        break;
    case zk::HASH_POSEIDON2: build<zk::HASH_POSEIDON2>(d, c, l, n_dig, n_cap, n_leaves, leaf_size, cap_height); break;
    case zk::HASH_MONOLITH: build<zk::HASH_MONOLITH>(d, c, l, n_dig, n_cap, n_leaves, leaf_size, cap_height); break;
    default: err = "unsupported hash_type " + std::to_string(hash_type); return false;
    }
    return true;
}

// host-side single hashes (used by the ABI's extension entry points)
bool zk_hash_one_cpu(uint64_t hash_type, const uint64_t *in, uint64_t n, uint64_t *out)
{
    switch (hash_type) {
    case zk::HASH_POSEIDON: zk::hash_one<zk::HASH_POSEIDON>(in, n, out); return true;
    case zk::HASH_KECCAK: zk::hash_one<zk::HASH_KECCAK>(in, n, out); return true;
    case zk::HASH_POSEIDON_BN128: zk::hash_one<zk::HASH_POSEIDON_BN128>(in, n, out); return true;
    case zk::HASH_POSEIDON2: zk::hash_one<zk::HASH_POSEIDON2>(in, n, out); return true;
    case zk::HASH_MONOLITH: zk::hash_one<zk::HASH_MONOLITH>(in, n, out); return true;
    default: return false;
    }
}

bool zk_hash_two_cpu(uint64_t hash_type, const uint64_t *l, const uint64_t *r, uint64_t *out)
{
    switch (hash_type) {
    case zk::HASH_POSEIDON: zk::hash_two<zk::HASH_POSEIDON>(l, r, out); return true;
    case zk::HASH_KECCAK: zk::hash_two<zk::HASH_KECCAK>(l, r, out); return true;
    case zk::HASH_POSEIDON_BN128: zk::hash_two<zk::HASH_POSEIDON_BN128>(l, r, out); return true;
    case zk::HASH_POSEIDON2: zk::hash_two<zk::HASH_POSEIDON2>(l, r, out); return true;
    case zk::HASH_MONOLITH: zk::hash_two<zk::HASH_MONOLITH>(l, r, out); return true;
    default: return false;
    }
}
