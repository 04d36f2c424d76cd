/*
 * int_types.h -- fixed-width aliases used by the zeknox headers
 * (drop-in for zeknox native/types/int_types.h:9-20).
 */
#ifndef ZEKNOX_TYPES_INT_TYPES_H
#define ZEKNOX_TYPES_INT_TYPES_H

#include <stdint.h>

typedef uint8_t u8;
typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;

#endif /* ZEKNOX_TYPES_INT_TYPES_H */
