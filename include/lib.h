/*
 * lib.h -- zeknox-compatible C ABI of the B200 Goldilocks commit library.
 *
 * Drop-in for zeknox native/lib.h (entry points defined in native/lib.cu):
 * the same names, argument meaning and error codes, so the Rust
 * (wrappers/rust/src/lib.rs:12-96) and Go (wrappers/go/lib/lib.go) bindings
 * link against libzeknox.a / libzeknox.so unchanged.  Each declaration cites
 * the reference definition it replaces.
 *
 * Threading: every entry point locks the device it works on; calls on one
 * device are serialised.  NTT/LDE/transpose calls are synchronous (they
 * return after the result is in place, like the reference's trailing sync).
 *
 * Tables: twiddle and coset tables are per device and built on first use;
 * init_* pre-builds them (the reference requires the init calls and crashes
 * without them).  The coset generator defaults to 7 until init_coset or
 * init_cuda_degree_and_generator sets another.
 */
#ifndef ZEKNOX_LIB_H
#define ZEKNOX_LIB_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#include "utils/rusterror.h"
#include "ntt/ntt.h"
#include "merkle/merkle.h"

#ifdef __cplusplus
#define ZK_EXTERN extern "C"
#else
#define ZK_EXTERN
#endif

/* native/lib.cu:65-70 -- number of CUDA devices. */
ZK_EXTERN RustError get_number_of_gpus(size_t *ngpus);

/* native/lib.cu:39-44 (utils/all_gpus.cu:150-184) -- print device properties. */
ZK_EXTERN RustError list_devices_info(void);

/* native/lib.cu:171-175 -- init_cuda_degree(24). */
ZK_EXTERN void init_cuda(void);

/* native/lib.cu:160-166 -- init_cuda_degree_and_generator(max_degree, 7). */
ZK_EXTERN void init_cuda_degree(const uint32_t max_degree);

/* native/lib.cu:140-155 -- on every GPU: coset powers of `group_generator` up to
 * 2^max_degree and the twiddle tables the transforms use. */
ZK_EXTERN void init_cuda_degree_and_generator(const uint32_t max_degree, const uint64_t group_generator);

/* native/lib.cu:118-123 (ntt/ntt.cu:160-173) -- forward and inverse twiddles of size 2^lg_n. */
ZK_EXTERN RustError init_twiddle_factors(size_t device_id, size_t lg_n);

/* native/lib.cu:128-133 (ntt/ntt.cu:228-239) -- coset generator and powers up to 2^lg_n. */
ZK_EXTERN RustError init_coset(size_t device_id, size_t lg_n, const uint64_t coset_gen);

/* native/lib.cu:75-81 (ntt/ntt.cu:253-309) -- in-place batched NTT of `batches`
 * columns of 2^lg_domain_size elements, natural order in and out.  Forward with
 * with_coset evaluates on g*H; inverse with with_coset multiplies the result
 * by g^i before the 1/n scaling (the reference's order).  inout is host or
 * device memory per cfg.are_inputs_on_device (both flags must agree). */
ZK_EXTERN RustError compute_batched_ntt(size_t device_id, void *inout, uint32_t lg_domain_size,
                                        NTT_Direction ntt_direction, NTT_Config cfg);

/* native/lib.cu:86-92 (ntt/ntt.cu:477-564) -- low-degree extension: input is
 * `batches` columns of 2^lg_domain_size coefficients, output `batches +
 * salt_size` columns of 2^(lg_domain_size + extension_rate_bits) evaluations
 * in natural order (on the coset g*H when with_coset).  lg_domain_size == 0 or
 * extension_rate_bits == 0 is rejected with cudaErrorInvalidValue. */
ZK_EXTERN RustError compute_batched_lde(size_t device_id, void *output, void *input, uint32_t lg_domain_size,
                                        NTT_Direction ntt_direction, NTT_Config cfg);

/* native/lib.cu:97-102 (ntt/ntt.cu:315-471) -- the same LDE with the columns
 * split across num_gpu GPUs; input on the host, output a device buffer on GPU 0
 * holding total_num_output_elements. */
ZK_EXTERN RustError compute_batched_lde_multi_gpu(void *output, void *input, uint32_t num_gpu,
                                                  NTT_Direction ntt_direction, NTT_Config cfg,
                                                  uint32_t lg_domain_size, size_t total_num_input_elements,
                                                  size_t total_num_output_elements);

/* native/lib.cu:107-113 (ntt/ntt.cu:182-226, kernels.cu:94-135) --
 * output[rev_lg_n(i) * batches + b] = input[b * 2^lg_n + i]. */
ZK_EXTERN RustError compute_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                          NTT_TransposeConfig cfg);

/* Declared at native/lib.h:50-51 but never defined by the reference; exported
 * here as the same operation as compute_transpose_rev. */
ZK_EXTERN RustError compute_naive_transpose_rev(size_t device_id, void *output, void *input, uint32_t lg_n,
                                                NTT_TransposeConfig cfg);

/* native/utils/all_gpus.cu:68 -- true when at least one CUDA device is present. */
ZK_EXTERN bool cuda_available(void);

#endif /* ZEKNOX_LIB_H */
