// Grid-wide barrier of the persistent propagation kernels (sparse_jacobi.cu,
// propagate.cu).  Every wait is bounded: a block that polls spin_limit times
// without seeing the barrier open raises the error flag, and every block that
// sees the flag leaves its kernel, so a bug cannot hang the GPU; the host
// reads the flag and reports IDL_ERR_INTERNAL.
#pragma once

#include <cuda/atomic>

namespace idl {

constexpr unsigned SPIN_LIMIT = 1u << 24;   // barrier polls before giving up

// Nanoseconds of the GPU's global timer (for per-pass profiling traces).
__device__ __forceinline__ unsigned long long global_timer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct GridSync {
    unsigned count;
    unsigned gen;
    int error;
    int passes;   // passes (or rounds) the kernel ran
    int last1;    // sparse kernel's round mode: last pass that changed a cell, plus one (0: none)
    int gens;     // sparse kernel: work-list generations it ran
};

__device__ __forceinline__ bool grid_sync(GridSync* gs, unsigned nblocks, unsigned& gen_local,
                                          unsigned spin_limit = SPIN_LIMIT)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(gs->count), gen(gs->gen);
        cuda::atomic_ref<int, cuda::thread_scope_device> err(gs->error);
        const unsigned target = gen_local + 1;
        int ok = 1;
        if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.store(target, cuda::memory_order_release);
        } else {
            unsigned spins = 0;
            while (gen.load(cuda::memory_order_acquire) != target) {
                if (++spins > spin_limit) {
                    err.fetch_or(1, cuda::memory_order_relaxed);
                    ok = 0;
                    break;
                }
                if (spins > 32) __nanosleep(20);
            }
        }
        if (err.load(cuda::memory_order_relaxed)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    ++gen_local;
    return s_ok != 0;
}

}  // namespace idl
