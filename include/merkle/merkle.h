/*
 * merkle.h -- linear-layout Merkle forest entry points.
 *
 * Drop-in for zeknox native/merkle/merkle.h:21-62.  Buffers: leaves is
 * leaves_buf_size rows of leaf_size u64 (leaf-major); digests has
 * digests_buf_size = 2 * (leaves_buf_size - cap_buf_size) slots of 4 u64; caps
 * has cap_buf_size = 2^cap_height slots of 4 u64.  Subtree k of the forest
 * owns digests [k(2L-2), (k+1)(2L-2)), L = leaves per subtree; inside it the
 * level with 2^r nodes starts at 2^r - 2 and the leaf digests at L - 2; the
 * subtree root is cap[k].  When cap_buf_size == leaves_buf_size the caps are the
 * leaf hashes and digests are not written.
 *
 * These functions return nothing (as in the reference).  On invalid sizes or an
 * unsupported hash they write nothing, print the reason to stderr and record
 * it for zeknox_last_error() (include/zeknox_b200.h).
 */
#ifndef ZEKNOX_MERKLE_MERKLE_H
#define ZEKNOX_MERKLE_MERKLE_H

#include <stdint.h>

#include "types/int_types.h"

#define HASH_SIZE 32
#define HASH_SIZE_U64 4

#ifdef __cplusplus
#define ZK_EXTERNC extern "C"
#else
#define ZK_EXTERNC
#endif

enum HashType { HashPoseidon = 0, HashKeccak = 1, HashPoseidonBN128 = 2, HashPoseidon2 = 3, HashMonolith = 4 };

/* GPU builder on device pointers of the current device
 * (replaces native/merkle/merkle.cu:246-280).  Work is queued on the legacy
 * default stream and not waited for, exactly like the reference: the results
 * are visible to later work on the default stream or on blocking streams. */
ZK_EXTERNC void fill_digests_buf_linear_gpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                         void *leaves_buf_gpu_ptr, u64 digests_buf_size,
                                                         u64 cap_buf_size, u64 leaves_buf_size, u64 leaf_size,
                                                         u64 cap_height, u64 hash_type, u64 gpu_id);

/* Multi-GPU builder, pointers on GPU 0: subtrees are split across the GPUs
 * (replaces native/merkle/merkle.cu:283-459).  Synchronous. */
ZK_EXTERNC void fill_digests_buf_linear_multigpu_with_gpu_ptr(void *digests_buf_gpu_ptr, void *cap_buf_gpu_ptr,
                                                              void *leaves_buf_gpu_ptr, u64 digests_buf_size,
                                                              u64 cap_buf_size, u64 leaves_buf_size, u64 leaf_size,
                                                              u64 cap_height, u64 hash_type);

/* Host builder on host pointers (replaces native/merkle/merkle.cpp:126-161). */
ZK_EXTERNC void fill_digests_buf_linear_cpu(void *digests_buf_ptr, void *cap_buf_ptr, const void *leaves_buf_ptr,
                                            u64 digests_buf_size, u64 cap_buf_size, u64 leaves_buf_size, u64 leaf_size,
                                            u64 cap_height, u64 hash_type);

/* Vector host builders, Poseidon only (replace native/merkle/merkle.h:64-88, which the
 * reference declares and exports only in USE_AVX / USE_AVX512 builds; always exported here).
 * Same forest as fill_digests_buf_linear_cpu; W = 8 (AVX-512) or 4 (AVX2) leaves per
 * permutation, the portable builder on CPUs without the instruction set. */
ZK_EXTERNC void fill_digests_buf_linear_cpu_avx(void *digests_buf_ptr, void *cap_buf_ptr, const void *leaves_buf_ptr,
                                                u64 digests_buf_size, u64 cap_buf_size, u64 leaves_buf_size,
                                                u64 leaf_size, u64 cap_height, u64 hash_type);
ZK_EXTERNC void fill_digests_buf_linear_cpu_avx512(void *digests_buf_ptr, void *cap_buf_ptr,
                                                   const void *leaves_buf_ptr, u64 digests_buf_size, u64 cap_buf_size,
                                                   u64 leaves_buf_size, u64 leaf_size, u64 cap_height, u64 hash_type);

#endif /* ZEKNOX_MERKLE_MERKLE_H */
