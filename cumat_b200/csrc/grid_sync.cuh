// Grid-wide barrier for cooperative launches (all CTAs co-resident, which
// cudaLaunchCooperativeKernel guarantees or refuses the launch).
//
// Two 64-bit words that only grow during a launch (zeroed before it):
// `arrive` counts arrivals, `release` the barriers completed. At its e-th
// barrier (e counted per CTA from 0) a CTA adds 1 to `arrive` with acq_rel
// semantics; the CTA that draws the value (e + 1) * G - 1 is the last to
// arrive. It runs a caller-supplied step with the whole CTA (the combine of
// the phase's per-CTA partial sums, so the scalars are computed once and in a
// fixed order) and then stores e + 1 to `release` with release semantics; the
// other CTAs poll `release` with acquire loads. No fence instructions are
// needed besides these, and the only serial chain per barrier is one atomic,
// the step, and one store seen by the pollers.
//
// The poll is bounded: a CTA that waits longer than the limit records
// DEVERR_GRID_BARRIER in the device error word and the barrier returns false,
// after which the caller leaves the kernel (the other CTAs then run out at
// their next barrier the same way). The limit is a launch argument
// (kGridBarrierSpins unless a test sets a short one), and so is a count of
// extra arrivals the barrier waits for (0; a test sets 1, an arrival that never
// comes, to make every CTA's wait run out).
//
// Data written before the barrier by other CTAs is read after it through L2
// (ld.global.cg / volatile), never through the non-coherent read-only path.
#pragma once

#include <cstdint>

namespace cmcg {

enum : int32_t { DEVERR_GRID_BARRIER = 2 };
constexpr long long kGridBarrierSpins = 1LL << 23;   // polls (with back-off, ~seconds) before giving up

struct GridSync {
    unsigned long long arrive;
    unsigned long long release;
};

__device__ __forceinline__ unsigned long long atom_add_acq_rel_gpu(unsigned long long* p, unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}

__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// epoch: this CTA's count of barriers passed (same in all CTAs), advanced here.
struct BarrierLimits {
    long long spins;        // polls before giving up
    unsigned extra;         // arrivals expected besides the grid's CTAs (0)
};

template <typename F>
__device__ __forceinline__ bool grid_barrier(GridSync* gs, int32_t* err, const BarrierLimits& lim,
                                             unsigned long long& epoch, F&& last_step) {
    __shared__ int s_last, s_ok;
    const unsigned long long target = epoch + 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        s_last = atom_add_acq_rel_gpu(&gs->arrive, 1ull) == target * (gridDim.x + lim.extra) - 1;
    }
    __syncthreads();
    if (s_last) {
        last_step();
        __syncthreads();
        if (threadIdx.x == 0) st_release_gpu(&gs->release, target);
    } else if (threadIdx.x == 0) {
        long long spins = 0;
        while (ld_acquire_gpu(&gs->release) < target) {
            if (++spins > lim.spins) {
                s_ok = 0;
                if (err) atomicOr(err, DEVERR_GRID_BARRIER);
                break;
            }
            __nanosleep(20);
        }
    }
    __syncthreads();
    epoch = target;
    return s_ok != 0;
}

}  // namespace cmcg
