/*
 * rusterror.h -- error value returned by the zeknox-compatible entry points.
 *
 * Drop-in for zeknox native/utils/rusterror.h:15-41: a {int code; char *message}
 * pair returned by value.  code == 0 is success; CUDA failures are the negated
 * cudaError_t, argument errors +cudaErrorInvalidValue (1).  message is NULL or a
 * malloc'd string that the caller releases with free() (the Rust wrapper's
 * Drop does, wrappers/rust/src/error.rs:11-17).  The reference declares C++
 * constructors on the struct; they are not part of the ABI and are omitted.
 */
#ifndef ZEKNOX_UTILS_RUSTERROR_H
#define ZEKNOX_UTILS_RUSTERROR_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct RustError {
    int code;
    char *message;
} RustError;

#ifdef __cplusplus
}
#endif

#endif /* ZEKNOX_UTILS_RUSTERROR_H */
