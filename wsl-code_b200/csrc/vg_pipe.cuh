// Shared-memory pipeline primitives for sm_100a (mbarrier + bulk copy PTX, sm_90+ forms): CTA-local
// transaction barriers, global -> shared bulk copies that complete on them, and a bounded wait.
#pragma once
#include "vg_common.cuh"

namespace vg {

constexpr unsigned long long WAIT_NS = 1000000000ull;  // 1 s: longer means a broken pipeline

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// L2 policy for data read once per apply (the operator records): evicted first, so the gathered
// x and the scattered y stay resident in L2 while the records stream through
__device__ __forceinline__ unsigned long long evict_first_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// global -> shared bulk copy into this CTA, completing on an mbarrier; 16-byte aligned, size % 16 == 0
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* b,
                                         unsigned long long pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(b)), "l"(pol)
        : "memory");
}

// the same without an L2 policy
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}

// order this thread's earlier generic-proxy accesses to shared memory before later bulk copies into it
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait for the phase of the given parity; false when it did not complete within WAIT_NS
// (or an iteration cap), or when abort (optional) was raised by another thread of the CTA
__device__ inline bool mbar_wait(unsigned long long* b, unsigned parity, const volatile int* abort) {
    if (mbar_try_wait(b, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (unsigned it = 1; it < (1u << 24); ++it) {
        if (mbar_try_wait(b, parity)) return true;
        if ((it & 31u) == 0) {
            if (abort && *abort) return false;
            if (globaltimer() - t0 > WAIT_NS) return false;
        }
    }
    return false;
}

// Programmatic dependent launch: a kernel launched with launch_pdl may start while the previous
// kernel in the stream is still running. It calls pdl_trigger() early (its own dependents may then
// launch once all of its CTAs have started) and pdl_wait() before it touches anything the previous
// kernel writes; before the wait it may only read data no earlier kernel of the chain modifies.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

#ifndef VG_PDL
#define VG_PDL 1  // 0: launch_pdl issues ordinary launches (the kernels' wait then returns at once)
#endif

template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = VG_PDL ? 1 : 0;
    VG_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

}  // namespace vg
