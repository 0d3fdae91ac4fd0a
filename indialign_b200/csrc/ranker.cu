// C ABI of the window ranker's training kernels: forward with saved
// activations, loss, backward and Adam on caller-owned device buffers.  No
// counterpart in the reference (it has no learned component).
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <string>

#include "../../include/indialign_b200.h"
#include "kernels.h"

namespace ia {

namespace {

static_assert(offsetof(MlpPacked, W2) % 16 == 0, "the packed W2 is a TMA source: 16-byte aligned");

constexpr size_t kAlign = 256;
size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
size_t rows16(int n) { return (size_t)((n + 15) / 16 * 16); }

// Save buffer: xn bf16 [n16][16] | z1 f32 [n16][128] | h1 bf16 [n16][128] | z2 f32 [n16][128]
MlpSave save_view(const void *base, int n) {
    const size_t r = rows16(n);
    char *p = static_cast<char *>(const_cast<void *>(base));
    MlpSave s;
    s.xn = reinterpret_cast<uint16_t *>(p);
    p += up(r * kFeatures * 2);
    s.z1 = reinterpret_cast<float *>(p);
    p += up(r * kHidden * 4);
    s.h1 = reinterpret_cast<uint16_t *>(p);
    p += up(r * kHidden * 2);
    s.z2 = reinterpret_cast<float *>(p);
    return s;
}
size_t save_bytes(int n) {
    const size_t r = rows16(n);
    return up(r * kFeatures * 2) + up(r * kHidden * 4) + up(r * kHidden * 2) + up(r * kHidden * 4);
}

constexpr int kSplitsMax = 64;
// Work buffer: dz2 bf16 [n16][128] | dh1 f32 [n16][128] | dz1 bf16 [n16][128] | split-K partials |
// row-block partial sums of the bias gradients
struct Work {
    uint16_t *dz2, *dz1;
    float *dh1, *part, *red;
};
Work work_view(void *base, int n) {
    const size_t r = rows16(n);
    char *p = static_cast<char *>(base);
    Work w;
    w.dz2 = reinterpret_cast<uint16_t *>(p);
    p += up(r * kHidden * 2);
    w.dh1 = reinterpret_cast<float *>(p);
    p += up(r * kHidden * 4);
    w.dz1 = reinterpret_cast<uint16_t *>(p);
    p += up(r * kHidden * 2);
    w.part = reinterpret_cast<float *>(p);
    p += up((size_t)kSplitsMax * kHidden * kHidden * 4);
    w.red = reinterpret_cast<float *>(p);
    return w;
}
size_t work_bytes(int n) {
    const size_t r = rows16(n);
    return up(r * kHidden * 2) + up(r * kHidden * 4) + up(r * kHidden * 2) +
           up((size_t)kSplitsMax * kHidden * kHidden * 4) + up((size_t)kBwdBlocksMax * kBwdRedStride * 4);
}

// K splits of a weight-gradient GEMM (K = batch rows): >= 256 rows per split.
int splits_for(int k) {
    const int s = k / 256;
    return s < 1 ? 1 : (s > kSplitsMax ? kSplitsMax : s);
}

int status(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return INDIALIGN_OK;
    set_last_error_text((std::string(what) + ": " + cudaGetErrorString(e)).c_str());
    return INDIALIGN_E_CUDA;
}

int bad(const char *what) {
    set_last_error_text(what);
    return INDIALIGN_E_INPUT;
}

}  // namespace

}  // namespace ia

extern "C" {

size_t indialign_mlp_packed_bytes(void) { return sizeof(ia::MlpPacked); }

size_t indialign_mlp_save_bytes(int n) { return n > 0 ? ia::save_bytes(n) : 0; }

size_t indialign_mlp_work_bytes(int n) { return n > 0 ? ia::work_bytes(n) : 0; }

int indialign_mlp_pack(const float *d_blob, void *d_packed, void *stream) {
    if (!d_blob || !d_packed) return ia::bad("mlp_pack: null pointer");
    ia::launch_mlp_pack(d_blob, static_cast<ia::MlpPacked *>(d_packed), static_cast<cudaStream_t>(stream));
    return ia::status("mlp_pack");
}

int indialign_mlp_forward(const void *d_packed, const float *d_x, int n, float *d_y, void *d_save,
                          void *stream) {
    if (n < 0 || (n > 0 && (!d_packed || !d_x || !d_y))) return ia::bad("mlp_forward: null pointer or n < 0");
    if (n == 0) return INDIALIGN_OK;
    ia::MlpSave sv = d_save ? ia::save_view(d_save, n) : ia::MlpSave{nullptr, nullptr, nullptr, nullptr};
    ia::launch_mlp_forward(static_cast<const ia::MlpPacked *>(d_packed), d_x, n, d_y, d_save ? &sv : nullptr,
                           static_cast<cudaStream_t>(stream));
    return ia::status("mlp_forward");
}

int indialign_mlp_loss(const float *d_y, const float *d_t, int n, float lambda, float *d_dy, float *d_loss,
                       void *stream) {
    if (n <= 0 || !d_y || !d_t || !d_dy || !d_loss) return ia::bad("mlp_loss: null pointer or n <= 0");
    ia::launch_mlp_loss(d_y, d_t, n, lambda, d_dy, d_loss, static_cast<cudaStream_t>(stream));
    return ia::status("mlp_loss");
}

int indialign_mlp_backward(const void *d_packed, const float *d_dy, int n, const void *d_save, float *d_grad,
                           void *d_work, void *stream) {
    using namespace ia;
    if (n <= 0 || !d_packed || !d_dy || !d_save || !d_grad || !d_work)
        return bad("mlp_backward: null pointer or n <= 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const MlpPacked *mlp = static_cast<const MlpPacked *>(d_packed);
    const MlpSave sv = save_view(d_save, n);
    const Work w = work_view(d_work, n);
    if (cudaMemsetAsync(d_grad, 0, kBlobW1 * sizeof(float), st) != cudaSuccess) return status("mlp_backward");
    // head: dz2, db2, dw3, db3
    launch_mlp_head_bwd(mlp, d_dy, sv.z2, n, w.dz2, w.red, d_grad, st);
    // The three products on the tcgen05 tensor cores, each operand read in
    // the layout it is stored in (h1, dz2, dz1, xn are [rows][features]:
    // MN-major for the weight gradients, K-major for dh1).
    int rc = 0;
    // dW2[i][j] = sum_r h1[r][i] dz2[r][j]   (M = N = 128, K = n, split over rows)
    rc |= launch_gemm_tc(sv.h1, kHidden, 1, w.dz2, kHidden, 1, kHidden, kHidden, n, d_grad + kBlobW2, kHidden, 0,
                         w.part, splits_for(n), nullptr, st);
    // dh1[r][i] = sum_j dz2[r][j] W2[i][j]   (W2 packed [in][out]: K-major B)
    const uint16_t *W2 = reinterpret_cast<const uint16_t *>(reinterpret_cast<const char *>(mlp) +
                                                            offsetof(MlpPacked, W2));
    rc |= launch_gemm_tc(w.dz2, kHidden, 0, W2, kHidden, 0, n, kHidden, kHidden, w.dh1, kHidden, 0, nullptr, 1,
                         nullptr, st);
    // dz1, db1
    launch_mlp_act_bwd(w.dh1, sv.z1, n, w.dz1, w.red, d_grad + kBlobB1, st);
    // dW1[f][i] = sum_r xn[r][f] dz1[r][i], computed as its transpose
    // (M = 128 hidden units on the TMEM lanes, N = 16 features) and stored transposed
    rc |= launch_gemm_tc(w.dz1, kHidden, 1, sv.xn, kFeatures, 1, kHidden, kFeatures, n, d_grad + kBlobW1, kHidden,
                         1, w.part, splits_for(n), nullptr, st);
    if (rc != 0) return bad("mlp_backward: tensor-core GEMM rejected its operands (alignment or tensor map)");
    return status("mlp_backward");
}

int indialign_gemm_bf16(const void *d_a, int lda, int a_mn, const void *d_b, int ldb, int b_mn, int m, int n,
                        int k, float *d_c, int ldc, int c_trans, float *d_partial, int splits, void *stream) {
    using namespace ia;
    const int rc = launch_gemm_tc(static_cast<const uint16_t *>(d_a), lda, a_mn ? 1 : 0,
                                  static_cast<const uint16_t *>(d_b), ldb, b_mn ? 1 : 0, m, n, k, d_c, ldc,
                                  c_trans ? 1 : 0, d_partial, splits, nullptr, static_cast<cudaStream_t>(stream));
    if (rc == -1) return bad("gemm_bf16: bad shape, stride, alignment or missing partial buffer");
    if (rc == -2) return bad("gemm_bf16: tensor map encoding failed");
    const int st = status("gemm_bf16");
    if (rc != 0 && st == INDIALIGN_OK) return bad("gemm_bf16: kernel attributes could not be set");
    return st;
}

int indialign_mlp_adam(float *d_blob, const float *d_grad, float *d_m, float *d_v, int step, float lr,
                       float beta1, float beta2, float eps, void *stream) {
    using namespace ia;
    if (!d_blob || !d_grad || !d_m || !d_v || step < 1) return bad("mlp_adam: null pointer or step < 1");
    const float bc1 = (float)(1.0 - std::pow((double)beta1, step));
    const float bc2 = (float)(1.0 - std::pow((double)beta2, step));
    launch_adam(d_blob, d_grad, d_m, d_v, kBlobSize, kBlobW1, lr, beta1, beta2, eps, bc1, bc2,
                static_cast<cudaStream_t>(stream));
    return status("mlp_adam");
}

}  // extern "C"
