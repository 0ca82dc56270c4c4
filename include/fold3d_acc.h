/*
 * fold3d_acc.h -- the subset of the OpenACC runtime API that the reference's
 * single-GPU host driver calls, implemented by libfold3dpmm.so over the CUDA
 * runtime:
 *   acc_malloc              AN_ISO_1_OpenACC.c:1185  (device field)
 *   acc_memcpy_to_device    AN_ISO_1_OpenACC.c:1186
 *   acc_memcpy_from_device  AN_ISO_1_OpenACC.c:1241
 *   acc_free                (the reference never frees the device field)
 * Prototypes as in OpenACC 2.x (openacc.h).  Do not include together with a
 * compiler's openacc.h in C++ (the exception specifications differ); C code
 * can include either.  acc_malloc records each allocation so that the
 * reference-compatible sweep functions, which take no grid size, can derive
 * the cube size from the allocation the field lives in.
 */
#ifndef FOLD3D_ACC_H
#define FOLD3D_ACC_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif
void *acc_malloc(size_t bytes);
void acc_free(void *p);
void acc_memcpy_to_device(void *dst, void *src, size_t bytes);
void acc_memcpy_from_device(void *dst, void *src, size_t bytes);
#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
