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
// Work buffer: dz2 bf16 [n16][128] | dh1 f32 [n16][128] | dz1 bf16 [n16][128] | split-K partials
struct Work {
    uint16_t *dz2, *dz1;
    float *dh1, *part;
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
    return w;
}
size_t work_bytes(int n) {
    const size_t r = rows16(n);
    return up(r * kHidden * 2) + up(r * kHidden * 4) + up(r * kHidden * 2) +
           up((size_t)kSplitsMax * kHidden * kHidden * 4);
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
    launch_mlp_head_bwd(mlp, d_dy, sv.z2, n, w.dz2, d_grad, st);
    // dW2 = h1^T dz2
    launch_gemm_bf16(sv.h1, 1, w.dz2, 0, kHidden, kHidden, n, d_grad + kBlobW2, w.part, splits_for(n), st);
    // dh1 = dz2 W2^T (W2 stored [in][out] = [n][k] of this product)
    const uint16_t *W2 = reinterpret_cast<const uint16_t *>(reinterpret_cast<const char *>(mlp) +
                                                            offsetof(MlpPacked, W2));
    launch_gemm_bf16(w.dz2, 0, W2, 1, n, kHidden, kHidden, w.dh1, w.part, 1, st);
    // dz1, db1
    launch_mlp_act_bwd(w.dh1, sv.z1, n, w.dz1, d_grad + kBlobB1, st);
    // dW1 = xn^T dz1
    launch_gemm_bf16(sv.xn, 1, w.dz1, 0, kFeatures, kHidden, n, d_grad + kBlobW1, w.part, splits_for(n), st);
    return status("mlp_backward");
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
