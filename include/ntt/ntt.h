/*
 * ntt.h -- configuration structs of the NTT / LDE / transpose entry points.
 *
 * Same layout as zeknox native/ntt/ntt.h:17-62 (the structs cross the FFI by
 * value): NTT_Config is 24 bytes, NTT_TransposeConfig 8 bytes; enums are int;
 * the boolean fields are one byte (bool in C++, char in C, as in the reference,
 * whose Go binding uses C and Rust binding C++).
 *
 * Field use (matches the reference): `order` and `ntt_type` are accepted and
 * ignored; `is_multi_gpu` is ignored by compute_batched_lde; `salt_size` adds
 * that many columns of random field elements after the LDE output.
 */
#ifndef ZEKNOX_NTT_NTT_H
#define ZEKNOX_NTT_NTT_H

#include <stdint.h>

#ifdef __cplusplus
#define ZK_BOOL bool
#else
#define ZK_BOOL char
#endif

typedef enum { NN, NR, RN, RR } NTT_InputOutputOrder;

typedef enum { forward, inverse } NTT_Direction;

typedef enum { standard, coset } NTT_Type;

typedef enum { GS, CT } NTT_Algorithm;

typedef struct {
    uint32_t batches;                /* number of columns (transforms) */
    NTT_InputOutputOrder order;      /* ignored: natural order in and out */
    NTT_Type ntt_type;               /* ignored */
    uint32_t extension_rate_bits;    /* LDE blowup = 2^extension_rate_bits */
    ZK_BOOL are_inputs_on_device;
    ZK_BOOL are_outputs_on_device;
    ZK_BOOL with_coset;              /* evaluate on the coset g*H (g from init_coset) */
    ZK_BOOL is_multi_gpu;            /* ignored */
    uint32_t salt_size;              /* extra random columns appended to the LDE output */
} NTT_Config;

typedef struct {
    uint32_t batches;
    ZK_BOOL are_inputs_on_device;
    ZK_BOOL are_outputs_on_device;
} NTT_TransposeConfig;

#undef ZK_BOOL

#endif /* ZEKNOX_NTT_NTT_H */
