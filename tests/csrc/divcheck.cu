// Test-only kernel: compares div_by_const (fold3d_fast.cuh) with CUDA's IEEE
// double division on the same operands, bit for bit.
#include <cstdint>

#include "fold3d_fast.cuh"

__global__ void divcheck_kernel(const double *x, const double *c, const double *r, long long n, int nc,
                                unsigned long long *mismatch, long long *first)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(i % nc);
        const double a = fold3d::div_by_const(x[i], c[j], r[j]);
        const double b = x[i] / c[j];
        if (__double_as_longlong(a) != __double_as_longlong(b)) {
            if (atomicAdd(mismatch, 1ull) == 0) *first = i;
        }
    }
}

extern "C" int divcheck(const double *x, const double *c, const double *r, long long n, int nc,
                        unsigned long long *mismatch, long long *first)
{
    divcheck_kernel<<<1184, 256>>>(x, c, r, n, nc, mismatch, first);
    return (int)cudaDeviceSynchronize();
}
