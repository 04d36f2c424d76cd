/* A C consumer of the static archive, linked the way zeknox's Rust build
 * (wrappers/rust/build.rs:107-114) links the reference: libzeknox.a + cudart
 * + libstdc++ + libgomp.  It runs the reference's commit sequence through the
 * reference's own entry points -- compute_batched_lde (host buffers) ->
 * compute_transpose_rev -> fill_digests_buf_linear_gpu_with_gpu_ptr -- and
 * prints the caps, one line of four hex words per cap.
 *
 * usage: consumer <lg_n> <rate_bits> <cols> <cap_height> <hash_type> <seed> */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "lib.h"
#include "merkle/merkle.h"

static uint64_t splitmix(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static int check(RustError e, const char *what)
{
    if (e.code) {
        fprintf(stderr, "%s failed: %d %s\n", what, e.code, e.message ? e.message : "");
        free(e.message);
        return 1;
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 7) return 2;
    const uint32_t lg = (uint32_t)atoi(argv[1]), rate = (uint32_t)atoi(argv[2]), cols = (uint32_t)atoi(argv[3]);
    const uint64_t cap = (uint64_t)atoi(argv[4]), hash = (uint64_t)atoi(argv[5]);
    uint64_t seed = (uint64_t)atoll(argv[6]);
    const uint64_t n = 1ULL << lg, N = n << rate, n_caps = 1ULL << cap;
    const uint64_t n_dig = n_caps < N ? 2 * (N - n_caps) : 0;
    uint64_t *coeffs = malloc(cols * n * 8), *evals = malloc(cols * N * 8), *caps = malloc(n_caps * 32);
    for (uint64_t i = 0; i < cols * n; i++) {
        uint64_t v = splitmix(&seed);
        coeffs[i] = v >= 0xFFFFFFFF00000001ULL ? v - 0xFFFFFFFF00000001ULL : v;
    }
    NTT_Config cfg = {0};
    cfg.batches = cols;
    cfg.extension_rate_bits = rate;
    cfg.with_coset = 1;
    if (check(compute_batched_lde(0, evals, coeffs, lg, forward, cfg), "compute_batched_lde")) return 1;
    uint64_t *d_evals, *d_leaves, *d_dig, *d_caps;
    if (cudaMalloc((void **)&d_evals, cols * N * 8) || cudaMalloc((void **)&d_leaves, cols * N * 8) ||
        cudaMalloc((void **)&d_dig, (n_dig ? n_dig : 1) * 32) || cudaMalloc((void **)&d_caps, n_caps * 32))
        return 1;
    cudaMemcpy(d_evals, evals, cols * N * 8, cudaMemcpyHostToDevice);
    NTT_TransposeConfig tcfg = {0};
    tcfg.batches = cols;
    tcfg.are_inputs_on_device = 1;
    tcfg.are_outputs_on_device = 1;
    if (check(compute_transpose_rev(0, d_leaves, d_evals, lg + rate, tcfg), "compute_transpose_rev")) return 1;
    fill_digests_buf_linear_gpu_with_gpu_ptr(d_dig, d_caps, d_leaves, n_dig, n_caps, N, cols, cap, hash, 0);
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    cudaMemcpy(caps, d_caps, n_caps * 32, cudaMemcpyDeviceToHost);
    for (uint64_t k = 0; k < n_caps; k++)
        printf("%016llx %016llx %016llx %016llx\n", (unsigned long long)caps[4 * k], (unsigned long long)caps[4 * k + 1],
               (unsigned long long)caps[4 * k + 2], (unsigned long long)caps[4 * k + 3]);
    return 0;
}
