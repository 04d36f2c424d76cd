/*
 * msm.h -- placeholder for zeknox native/msm/msm.h.
 *
 * The Go binding includes this header unconditionally
 * (wrappers/go/lib/lib.go:11).  BN254 multi-scalar multiplication is not part
 * of this library (it is not on the Goldilocks commit path), so the header
 * declares nothing; it exists so that consumers keep compiling.
 */
#ifndef ZEKNOX_MSM_MSM_H
#define ZEKNOX_MSM_MSM_H
#endif /* ZEKNOX_MSM_MSM_H */
