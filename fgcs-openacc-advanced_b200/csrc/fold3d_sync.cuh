// fold3d_sync.cuh -- device helpers of the persistent tile-dataflow kernels
// (forward passes in fold3d_wavefront.cu, backward passes in
// fold3d_adjoint.cu): gpu-scope acquire loads and release stores of the
// completion flags, and the global nanosecond timer that bounds every wait.
#pragma once

namespace fold3d {

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace fold3d
