// FP64 and FP32 pipe throughput probes: the denominators of the search
// kernels' rooflines.  The search is SIMT work (FP64 score matrices, NW and
// Kabsch; FP32 seed-bank residue visits); it uses neither HBM bandwidth nor
// tensor cores to any extent, so its ceiling is the FMA rate of the SMs,
// measured here with independent FMA chains (8 per thread, enough to hide
// FMA latency at full occupancy).
#include <cuda_runtime.h>

#include "../../include/indialign_b200.h"
#include "dmath.cuh"

namespace ia {

template <typename T>
__global__ void k_fma_chains(T *out, int iters, T a, T b) {
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    T x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; i++) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)12345.678) out[0] = s;  // keeps the chains live
}

// Best of 5 timed launches of 8 independent FMA chains per thread.
template <typename T>
static int fma_peak(int device, double *tflops) {
    if (!tflops) return INDIALIGN_E_INPUT;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return INDIALIGN_E_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device < 0 ? 0 : device) != cudaSuccess)
        return INDIALIGN_E_CUDA;
    T *d = nullptr;
    if (cudaMalloc(&d, 64) != cudaSuccess) return INDIALIGN_E_CUDA;
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    const T a = (T)0.999999, b = (T)1e-7;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_chains<T><<<blocks, threads>>>(d, iters / 8, a, b);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0);
        k_fma_chains<T><<<blocks, threads>>>(d, iters, a, b);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (e != cudaSuccess) return INDIALIGN_E_CUDA;
    *tflops = 2.0 * 8.0 * (double)iters * blocks * threads / (best * 1e-3) / 1e12;
    return INDIALIGN_OK;
}

}  // namespace ia

extern "C" int indialign_fp64_peak(int device, double *tflops) { return ia::fma_peak<double>(device, tflops); }

extern "C" int indialign_fp32_peak(int device, double *tflops) { return ia::fma_peak<float>(device, tflops); }

namespace ia {
__global__ void k_rcp_check(const double *x, double *y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = rcp_nr(x[i]);
}
}  // namespace ia

// Diagnostic: the search's Newton-Raphson reciprocal on the device for n
// host values (tests compare it with the correctly rounded 1/x).
extern "C" int indialign_selftest_rcp(int n, const double *x, double *y) {
    if (n <= 0 || !x || !y) return INDIALIGN_E_INPUT;
    double *d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(double) * (size_t)n) != cudaSuccess) return INDIALIGN_E_CUDA;
    cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    ia::k_rcp_check<<<(n + 255) / 256, 256>>>(d, d + n, n);
    cudaError_t e = cudaMemcpy(y, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? INDIALIGN_OK : INDIALIGN_E_CUDA;
}

namespace ia {
__global__ void k_rotation_check(const double *H9, double *R9, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double H[3][3];
#pragma unroll
    for (int a = 0; a < 9; a++) H[a / 3][a % 3] = H9[9 * (size_t)i + a];
    double R[9];
    cov_to_rotation(H, R);
#pragma unroll
    for (int a = 0; a < 9; a++) R9[9 * (size_t)i + a] = R[a];
}
}  // namespace ia

// Diagnostic: the search's eigen-solve on the device for n host covariances
// (tests compare it with the reference's rotation).
extern "C" int indialign_selftest_rotation(int n, const double *H, double *R) {
    if (n <= 0 || !H || !R) return INDIALIGN_E_INPUT;
    double *d = nullptr;
    const size_t bytes = 9 * sizeof(double) * (size_t)n;
    if (cudaMalloc(&d, 2 * bytes) != cudaSuccess) return INDIALIGN_E_CUDA;
    cudaError_t e = cudaMemcpy(d, H, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        ia::k_rotation_check<<<(n + 127) / 128, 128>>>(d, d + 9 * (size_t)n, n);
        e = cudaMemcpy(R, d + 9 * (size_t)n, bytes, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    return e == cudaSuccess ? INDIALIGN_OK : INDIALIGN_E_CUDA;
}
