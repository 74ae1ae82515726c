// treesap-b200 engine: thin inline-PTX wrappers for sm_100a (mbarrier, TMA bulk tensor
// loads, proxy fences, the global timer). Every wait is bounded: after `kWaitLimitNs` it
// records an error bit in the context's device error word and reports failure, so a lost
// transfer can never hang the GPU.
#pragma once

#include <cstdint>
#include <cuda.h>

namespace treesap_b200 {

/// Device error bits (OR-ed into the context's error word; read by ts_context_sync()).
enum DeviceError : int {
    kErrMbarTimeout = 1, // a bounded mbarrier wait expired (TMA data never arrived)
    kErrBounds = 2,      // a checked index was out of range (bounds-checked builds)
    kErrBadLaunch = 4    // a kernel found an inconsistent launch configuration
};

constexpr unsigned long long kWaitLimitNs = 2000000000ull; // 2 s
/// Wait bound of a launch that carries an injected fault (ts_context_inject_fault).
constexpr unsigned long long kInjectedWaitLimitNs = 1000000ull; // 1 ms

/// Records `bit` in a device error word (atomically on the device; plain OR on the host).
__host__ __device__ __forceinline__ void flag_error(int* err, int bit) {
    if (!err) return;
#if defined(__CUDA_ARCH__)
    atomicOr(err, bit);
#else
    *err |= bit;
#endif
}

namespace ptx {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

/// Arrives on `bar` when `pred` holds (predicated, no branch): the elected lane of a warp
/// releasing a ring slot after __syncwarp().
__device__ __forceinline__ void mbar_arrive_if(uint64_t* bar, bool pred) {
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %1, 0;\n\t"
                 "@p mbarrier.arrive.shared::cta.b64 _, [%0];\n\t}" ::"r"(smem_addr(bar)),
                 "r"(int(pred))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}

/// Waits for phase `parity` of `bar` to complete; false (and error bit set) after kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          unsigned long long limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer() - t0 > limit_ns) {
            if (err) atomicOr(err, kErrMbarTimeout);
            return false;
        }
    }
}

/// 4-d tiled TMA load of one box into this CTA's own shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void prefetch_tensor_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

} // namespace ptx
} // namespace treesap_b200
