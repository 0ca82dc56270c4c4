// fold3d_sync.cuh -- device helpers of the persistent tile-dataflow kernels
// (forward passes in fold3d_wavefront.cu, backward passes in
// fold3d_adjoint.cu): gpu-scope acquire loads and release stores of the
// completion flags, the global nanosecond timer that bounds every wait, and
// the item lookup of batched launches.
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

// Batched launches order their items step-major across instances (step p of
// every instance that has one, then step p+1; instances sorted by their
// number of steps, so the active ones of a step are a prefix).  Locates
// global item gitem: its instance slot il and the item's number within that
// instance's own pass (step * tiles + tile).
__device__ __forceinline__ void batch_locate(const long long *step_off, const int *step_k, const long long *tile_pre,
                                             int max_steps, long long gitem, int &il, int &local)
{
    int lo = 0, hi = max_steps;  // step_off[lo] <= gitem < step_off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (step_off[mid] <= gitem) lo = mid; else hi = mid;
    }
    const long long r = gitem - step_off[lo];
    int a = 0, b = step_k[lo];
    while (b - a > 1) {
        const int mid = (a + b) >> 1;
        if (tile_pre[mid] <= r) a = mid; else b = mid;
    }
    il = a;
    local = lo * (int)(tile_pre[a + 1] - tile_pre[a]) + (int)(r - tile_pre[a]);
}

}  // namespace fold3d
