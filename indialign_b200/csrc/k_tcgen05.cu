// BF16 GEMM on the 5th-generation tensor cores (tcgen05) for the ranker's
// training backward:  C[M x N] (FP32) = A[M x K] . B[N x K]^T.
//
// Operands stay in the layouts the forward and backward kernels write; each
// is either K-major (row-major [rows][K], K contiguous) or MN-major
// (row-major [K][rows], the M or N index contiguous), and the tensor cores
// read either from shared memory through the matrix descriptor:
//
//   K-major slab  : box {64 K, rows} -> rows x 128 B, 128-byte swizzle;
//                   8-row groups 1024 B apart (SBO), the K = 16 slice of MMA
//                   step kk starts 32 kk bytes into each row.
//   MN-major slab : boxes {64 rows, 64 K} -> 64 K-rows x 128 B each, 128-byte
//                   swizzle, 8192 B apart (LBO between 64-wide MN blocks);
//                   8-K-row groups 1024 B apart (SBO); MMA step kk starts
//                   2048 kk bytes in.
//
// One CTA of 128 threads computes a 128-row x N tile (N <= 256) over a K
// range (split-K over gridDim.z writes partial tiles that k_splitk_sum_tc
// adds in a fixed order).  Thread 0 runs a two-stage ring: TMA
// (cp.async.bulk.tensor, this GPU's own memory, no multicast) loads 64-wide
// K slabs of A and B into a stage, completion on that stage's `full`
// mbarrier; four tcgen05.mma (kind::f16: BF16 in, FP32 accumulate, M = 128,
// K = 16 each) per slab accumulate into a TMEM tile of 128 lanes x N
// columns; tcgen05.commit arrives on the stage's `done` mbarrier when the
// MMAs have finished reading it, which frees the stage for the slab after
// next.  After the last slab every warp reads its 32 TMEM lanes (rows) with
// tcgen05.ld and stores them (optionally transposed).
//
// Every mbarrier wait is bounded.  On a timeout the CTA records
// DERR_TMA_TIMEOUT, gives the copies and MMAs in flight a second bounded
// wait, writes NaN over its output tile (so the loss and gradients show the
// failure), and still frees its TMEM columns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cmath>
#include <mutex>

#include "dmath.cuh"
#include "kernels.h"
#include "stage.cuh"

namespace ia {

namespace {

constexpr int kTcBK = 64;        // K elements per slab: one 128-byte swizzle row of BF16
constexpr int kTcBM = 128;       // rows of the M tile = TMEM lanes
constexpr int kTcStages = 2;
constexpr uint32_t kTcABytes = kTcBM * 128;  // A slab: 128 rows (or 2 MN boxes of 64 K-rows) x 128 B

// Shared-memory matrix descriptor, 128-byte swizzle (sm_100 format:
// start >> 4 in [0,14), LBO >> 4 in [16,30), SBO >> 4 in [32,46), version 1
// at bit 46, layout type 2 = SWIZZLE_128B in [61,64)).
IA_DEV uint64_t sw128_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Instruction descriptor of kind::f16: D FP32 (bits [4,6) = 1), A and B BF16
// ([7,10) = [10,13) = 1), A / B major at bits 15 / 16 (1 = MN-major),
// N >> 3 in [17,23), M >> 4 in [24,29).
IA_DEV uint32_t idesc_bf16(int nmma, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(nmma >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
}

IA_DEV void tma_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

IA_HD_INLINE uint32_t b_slab_bytes(int nmma, int b_mn) {
    return b_mn ? (uint32_t)(nmma / 64) * 8192u : (uint32_t)nmma * 128u;
}

}  // namespace

struct TcArgs {
    int M, N, nmma, K, kper, a_mn, b_mn;
    float *out;           // split z writes out + z * split_stride
    size_t split_stride;
    int ldo, trans;
    uint32_t tmem_cols;
    int *err;
};

__global__ void __launch_bounds__(128, 1)
k_gemm_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TcArgs a) {
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    __shared__ uint64_t full[kTcStages], done[kTcStages];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    unsigned char *base =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t stage_bytes = kTcABytes + b_slab_bytes(a.nmma, a.b_mn);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kTcBM;
    const int kbeg = blockIdx.z * a.kper;
    const int kend = min(a.K, kbeg + a.kper);
    const int nslab = kend > kbeg ? (kend - kbeg + kTcBK - 1) / kTcBK : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcStages; s++) {
            mbar_init(&full[s]);
            mbar_init(&done[s]);
        }
        failed = 0;
    }
    if (warp == 0) {  // the whole warp allocates the accumulator columns, then gives up the permit
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(a.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (threadIdx.x == 0) {
        const uint32_t idesc = idesc_bf16(a.nmma, a.a_mn, a.b_mn);
        auto load = [&](int i) {
            const int s = i & 1, k0 = kbeg + i * kTcBK;
            unsigned char *sa = base + s * stage_bytes, *sb = sa + kTcABytes;
            mbar_expect_tx(&full[s], stage_bytes);
            if (a.a_mn) {
                tma_2d(sa, &tmA, m0, k0, &full[s]);
                tma_2d(sa + 8192, &tmA, m0 + 64, k0, &full[s]);
            } else {
                tma_2d(sa, &tmA, k0, m0, &full[s]);
            }
            if (a.b_mn) {
                for (int b = 0; b < a.nmma / 64; b++) tma_2d(sb + 8192 * b, &tmB, 64 * b, k0, &full[s]);
            } else {
                tma_2d(sb, &tmB, k0, 0, &full[s]);
            }
        };
        // loaded: slabs whose copies were issued; landed: slabs whose copies
        // completed; issued: slabs whose MMAs were committed
        int loaded = 0, landed = 0, issued = 0;
        bool ok = true;
        if (nslab > 0) load(loaded++);
        for (int i = 0; i < nslab && ok; i++) {
            const int s = i & 1;
            if (i + 1 < nslab) {
                // stage (i+1)&1 last held slab i-1: wait for its MMAs to finish reading it
                if (i >= 1 && !mbar_wait(&done[(i + 1) & 1], ((i - 1) >> 1) & 1)) {
                    ok = false;
                    break;
                }
                load(loaded++);
            }
            if (!mbar_wait(&full[s], (i >> 1) & 1)) {
                ok = false;
                break;
            }
            landed++;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(base + s * stage_bytes), sb = sa + kTcABytes;
#pragma unroll
            for (int kk = 0; kk < kTcBK / 16; kk++) {
                const uint64_t da = a.a_mn ? sw128_desc(sa + 2048u * kk, 8192u, 1024u)
                                           : sw128_desc(sa + 32u * kk, 16u, 1024u);
                const uint64_t db = a.b_mn ? sw128_desc(sb + 2048u * kk, 8192u, 1024u)
                                           : sw128_desc(sb + 32u * kk, 16u, 1024u);
                const uint32_t acc = (i > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&done[s]))
                         : "memory");
            issued++;
        }
        // copies still in flight after a timeout get one more bounded wait each
        for (int j = landed; j < loaded; j++) mbar_wait(&full[j & 1], (j >> 1) & 1);
        // the commit of the last slab issued covers every MMA before it
        if (issued > 0) {
            const int j = issued - 1;
            if (!mbar_wait(&done[j & 1], (j >> 1) & 1)) {
                ok = false;
                mbar_wait(&done[j & 1], (j >> 1) & 1);
            }
        }
        if (!ok) {
            failed = 1;
            if (a.err) atomicOr(a.err, DERR_TMA_TIMEOUT);
        } else if (nslab == 0) {
            failed = 2;  // empty K range: the tile is zero
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = m0 + warp * 32 + lane;
    float *const out = a.out + (size_t)blockIdx.z * a.split_stride;
    const int fl = failed;
    const float fill = fl == 1 ? __int_as_float(0x7fc00000) : 0.f;
    const bool vec = !a.trans && (a.ldo & 3) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    for (int c0 = 0; c0 < a.N; c0 += 16) {
        uint32_t v[16];
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
            "%13, %14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row >= a.M) continue;
        float f[16];
#pragma unroll
        for (int j = 0; j < 16; j++) f[j] = fl ? fill : __uint_as_float(v[j]);
        if (vec && c0 + 16 <= a.N) {
            float4 *o = reinterpret_cast<float4 *>(out + (size_t)row * a.ldo + c0);
#pragma unroll
            for (int q = 0; q < 4; q++) o[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int col = c0 + j;
                if (col < a.N) {
                    if (a.trans) out[(size_t)col * a.ldo + row] = f[j];
                    else out[(size_t)row * a.ldo + col] = f[j];
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols)
                     : "memory");
}

// C (row stride ldo, or transposed) = sum over z of part[z][M][N], in z order.
__global__ void k_splitk_sum_tc(const float *__restrict__ part, int splits, int M, int N, float *C, int ldo,
                                int trans) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M * N) return;
    float s = 0.f;
    for (int z = 0; z < splits; z++) s += part[(size_t)z * M * N + i];
    const int r = i / N, c = i % N;
    if (trans) C[(size_t)c * ldo + r] = s;
    else C[(size_t)r * ldo + c] = s;
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

// Tensor map of a row-major BF16 matrix [outer][ld] whose first `inner`
// columns are the data, boxes {box_inner, box_outer}, 128-byte swizzle;
// elements outside [0, inner) x [0, outer) load as zero.
bool make_map(CUtensorMap *map, const void *ptr, int inner, int outer, int ld, int box_inner, int box_outer) {
    std::call_once(g_encode_once, []() {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
    const cuuint32_t estr[2] = {1, 1};
    return g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int nmma_of(int N, int b_mn) { return b_mn ? (N + 63) / 64 * 64 : (N + 15) / 16 * 16; }

}  // namespace

size_t gemm_tc_smem_bytes(int N, int b_mn) {
    return 1024 + (size_t)kTcStages * (kTcABytes + b_slab_bytes(nmma_of(N, b_mn), b_mn));
}

namespace {

// The kernel's dynamic shared-memory limit, raised once per device.
bool ensure_attributes() {
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    const uint64_t bit = 1ull << dev;
    if (done.load() & bit) return true;
    if (cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_tc_smem_bytes(256, 1)) != cudaSuccess)
        return false;
    done.fetch_or(bit);
    return true;
}

}  // namespace

int launch_gemm_tc(const uint16_t *A, int lda, int a_mn, const uint16_t *B, int ldb, int b_mn, int M, int N, int K,
                   float *C, int ldc, int c_trans, float *partial, int splits, int *err, cudaStream_t st) {
    if (M < 1 || N < 1 || N > 256 || K < 1 || lda % 8 || ldb % 8 || !A || !B || !C) return -1;
    if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15)) return -1;
    if (a_mn ? (M > kTcBM || lda < M) : lda < K) return -1;  // an MN-major A is one 128-row tile
    if (b_mn ? ldb < N : ldb < K) return -1;
    // output rows may not overlap, and the split-K sum indexes M x N in int
    if (ldc < (c_trans ? M : N) || (long long)M * N > 0x7fffffffLL) return -1;
    const int nmma = nmma_of(N, b_mn);
    CUtensorMap ma, mb;
    const bool okA = a_mn ? make_map(&ma, A, M, K, lda, 64, kTcBK) : make_map(&ma, A, K, M, lda, kTcBK, kTcBM);
    const bool okB = b_mn ? make_map(&mb, B, N, K, ldb, 64, kTcBK) : make_map(&mb, B, K, N, ldb, kTcBK, nmma);
    if (!okA || !okB) return -2;
    if (!ensure_attributes()) return -3;
    if (splits < 1) splits = 1;
    int kper = (K + splits - 1) / splits;
    kper = (kper + kTcBK - 1) / kTcBK * kTcBK;
    splits = (K + kper - 1) / kper;
    if (splits > 1 && !partial) return -1;
    uint32_t cols = 32;
    while ((int)cols < nmma) cols <<= 1;
    TcArgs t{M, N, nmma, K, kper, a_mn, b_mn, C, 0, ldc, c_trans, cols, err};
    if (splits > 1) {
        t.out = partial;
        t.split_stride = (size_t)M * N;
        t.ldo = N;
        t.trans = 0;
    }
    const dim3 grid((M + kTcBM - 1) / kTcBM, 1, splits);
    k_gemm_tc<<<grid, 128, gemm_tc_smem_bytes(N, b_mn), st>>>(ma, mb, t);
    if (splits > 1) k_splitk_sum_tc<<<(M * N + 255) / 256, 256, 0, st>>>(partial, splits, M, N, C, ldc, c_trans);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace ia
