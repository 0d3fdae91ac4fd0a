// Shared-memory staging helpers: bulk (TMA engine) global->shared copies
// completed on an mbarrier, with bounded waits, and a plain-load fallback
// for ranges the bulk engine cannot take (unaligned or odd sizes).
#pragma once
#include <stdint.h>
#include "pipeline.h"

namespace ia {

constexpr uint32_t kWaitLimit = 1u << 24;  // try_wait polls before giving up

IA_DEV uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

IA_DEV void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

IA_DEV void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bounded wait on the given phase parity; returns false on timeout.
IA_DEV bool mbar_wait(uint64_t *bar, uint32_t parity) {
    uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

IA_DEV void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

IA_DEV void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// A planned copy of `bytes` bytes at `src` into a 16-byte aligned shared
// region.  The bulk engine needs 16-byte aligned source, destination and
// size, so the source is rounded down to 16 bytes and the size up; the data
// then starts `lead` bytes into the region.  Device buffers carry >= 16 bytes
// of tail padding so the rounded-up read stays inside the allocation.
struct Copy {
    const char *src;
    uint32_t bytes;
    uint32_t lead;
};

IA_DEV Copy plan_copy(const void *src, uint32_t bytes) {
    uintptr_t s = reinterpret_cast<uintptr_t>(src);
    uintptr_t a = s & ~uintptr_t(15);
    Copy c;
    c.src = reinterpret_cast<const char *>(a);
    c.lead = static_cast<uint32_t>(s - a);
    c.bytes = (c.lead + bytes + 15u) & ~15u;
    return c;
}

// CTA-wide: issue the planned copies (thread 0) and wait for all of them.
// Copies whose shapes the bulk engine cannot take are done with plain loads.
// `phase` is the barrier's current parity and flips on every use.
IA_DEV void stage_copies(const Copy *cp, char *const *dst, int ncopies,
                         uint64_t *bar, uint32_t &phase, int *err) {
    bool bulk_ok = true;
    uint32_t total = 0;
    for (int i = 0; i < ncopies; i++) {
        uintptr_t d = reinterpret_cast<uintptr_t>(dst[i]);
        bulk_ok &= ((d & 15u) == 0) && ((cp[i].bytes & 15u) == 0) &&
                   ((reinterpret_cast<uintptr_t>(cp[i].src) & 15u) == 0);
        total += cp[i].bytes;
    }
    if (bulk_ok && total > 0) {
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_proxy_async();
            mbar_expect_tx(bar, total);
            for (int i = 0; i < ncopies; i++)
                if (cp[i].bytes) bulk_g2s(dst[i], cp[i].src, cp[i].bytes, bar);
        }
        if (!mbar_wait(bar, phase)) {
            atomicOr(err, DERR_TMA_TIMEOUT);
            mbar_wait(bar, phase);  // give in-flight copies a second bounded chance
        }
        phase ^= 1u;
        __syncthreads();
    } else {
        __syncthreads();
        for (int i = 0; i < ncopies; i++) {
            const char *s = cp[i].src;
            for (uint32_t b = threadIdx.x; b < cp[i].bytes; b += blockDim.x) dst[i][b] = s[b];
        }
        __syncthreads();
    }
}

}  // namespace ia
