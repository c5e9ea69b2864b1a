// Training and packing of the early-termination network: 12 -> 64 -> 64 -> 1, ReLU.
//
// The network has no reference counterpart (it is the learned part of this engine). Training keeps
// float32 master weights and runs the forward pass with BF16-rounded weights and FP32
// accumulation -- exactly the arithmetic of the in-search inference (search.cu, mlp_eval) -- so the
// trained network behaves identically when it is packed and used by the search kernel.
//
// Master parameter vector (float32, MLP_PARAMS values):
//   W1 [64][12] | b1 [64] | W2 [64][64] | b2 [64] | W3 [64] | b3 [1]
// Loss: mean squared error of the prediction against log1p(remaining checkpoints).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "hnsw_b200.h"

namespace hb {
int fail(int code, const std::string &msg);
}

namespace hbm {

constexpr int F = HNSW_B200_STOP_FEATURES;  // 12
constexpr int H = HNSW_B200_STOP_HIDDEN;    // 64
constexpr int O_W1 = 0;
constexpr int O_B1 = O_W1 + H * F;
constexpr int O_W2 = O_B1 + H;
constexpr int O_B2 = O_W2 + H * H;
constexpr int O_W3 = O_B2 + H;
constexpr int O_B3 = O_W3 + H;
constexpr int NPARAM = O_B3 + 1;  // 5057
constexpr unsigned FULL = 0xffffffffu;
// Shared-memory copy with padded row strides (13 and 65 words) so that lane j reading row j is
// bank-conflict free.
constexpr int S_W1 = 13, S_W2 = 65;
constexpr int SMEM_FLOATS = H * S_W1 + H + H * S_W2 + H + H + 1;

__device__ __forceinline__ float bf(float w) { return __bfloat162float(__float2bfloat16_rn(w)); }

__device__ void load_weights(const float *P, float *s) {
    float *w1 = s, *b1 = w1 + H * S_W1, *w2 = b1 + H, *b2 = w2 + H * S_W2, *w3 = b2 + H, *b3 = w3 + H;
    for (int i = threadIdx.x; i < H * F; i += blockDim.x) w1[(i / F) * S_W1 + i % F] = bf(P[O_W1 + i]);
    for (int i = threadIdx.x; i < H * H; i += blockDim.x) w2[(i / H) * S_W2 + i % H] = bf(P[O_W2 + i]);
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        b1[i] = P[O_B1 + i];
        b2[i] = P[O_B2 + i];
        w3[i] = bf(P[O_W3 + i]);
    }
    if (threadIdx.x == 0) b3[0] = P[O_B3];
    __syncthreads();
}

// Forward of one sample by one warp: h1 (lanes j, j+32), h2 (lanes j, j+32), output (all lanes).
__device__ __forceinline__ float forward(const float *s, const float *x, int lane, float &h1a,
                                         float &h1b, float &h2a, float &h2b) {
    const float *w1 = s, *b1 = w1 + H * S_W1, *w2 = b1 + H, *b2 = w2 + H * S_W2, *w3 = b2 + H, *b3 = w3 + H;
    h1a = b1[lane];
    h1b = b1[lane + 32];
#pragma unroll
    for (int i = 0; i < F; i++) {
        h1a = fmaf(w1[lane * S_W1 + i], x[i], h1a);
        h1b = fmaf(w1[(lane + 32) * S_W1 + i], x[i], h1b);
    }
    h1a = fmaxf(h1a, 0.f);
    h1b = fmaxf(h1b, 0.f);
    h2a = b2[lane];
    h2b = b2[lane + 32];
#pragma unroll 8
    for (int i = 0; i < 32; i++) {
        const float u = __shfl_sync(FULL, h1a, i), v = __shfl_sync(FULL, h1b, i);
        h2a = fmaf(w2[lane * S_W2 + i], u, h2a);
        h2b = fmaf(w2[(lane + 32) * S_W2 + i], u, h2b);
        h2a = fmaf(w2[lane * S_W2 + 32 + i], v, h2a);
        h2b = fmaf(w2[(lane + 32) * S_W2 + 32 + i], v, h2b);
    }
    h2a = fmaxf(h2a, 0.f);
    h2b = fmaxf(h2b, 0.f);
    float o = w3[lane] * h2a + w3[lane + 32] * h2b;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) o += __shfl_xor_sync(FULL, o, off);
    return o + b3[0];
}

// Per-sample forward and backward: activations and their gradients for the reduction kernel.
__global__ void mlp_fwd_bwd(const float *P, const float *X, const float *Y, int B, float *H1,
                            float *H2, float *dH1, float *dH2, float *dO, float *loss) {
    extern __shared__ float sw[];
    load_weights(P, sw);
    const float *w2 = sw + H * S_W1 + H, *w3 = w2 + H * S_W2 + H;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    float lsum = 0.f;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < B; b += warps) {
        float x[F];
#pragma unroll
        for (int i = 0; i < F; i++) x[i] = X[int64_t(b) * F + i];
        float h1a, h1b, h2a, h2b;
        const float o = forward(sw, x, lane, h1a, h1b, h2a, h2b);
        const float err = o - Y[b];
        const float g = 2.f * err / float(B);
        lsum += err * err / float(B);
        const float g2a = h2a > 0.f ? g * w3[lane] : 0.f;
        const float g2b = h2b > 0.f ? g * w3[lane + 32] : 0.f;
        // dh1[i] = sum_j W2[j][i] dh2[j]; lane i holds i and i + 32.
        float g1a = 0.f, g1b = 0.f;
#pragma unroll 8
        for (int j = 0; j < 32; j++) {
            const float u = __shfl_sync(FULL, g2a, j), v = __shfl_sync(FULL, g2b, j);
            g1a = fmaf(w2[j * S_W2 + lane], u, g1a);
            g1b = fmaf(w2[j * S_W2 + lane + 32], u, g1b);
            g1a = fmaf(w2[(j + 32) * S_W2 + lane], v, g1a);
            g1b = fmaf(w2[(j + 32) * S_W2 + lane + 32], v, g1b);
        }
        g1a = h1a > 0.f ? g1a : 0.f;
        g1b = h1b > 0.f ? g1b : 0.f;
        const int64_t r = int64_t(b) * H;
        H1[r + lane] = h1a;
        H1[r + lane + 32] = h1b;
        H2[r + lane] = h2a;
        H2[r + lane + 32] = h2b;
        dH1[r + lane] = g1a;
        dH1[r + lane + 32] = g1b;
        dH2[r + lane] = g2a;
        dH2[r + lane + 32] = g2b;
        if (lane == 0) dO[b] = g;
    }
    if (lane == 0 && lsum != 0.f) atomicAdd(loss, lsum);
}

// Weight gradients: one thread per parameter, summed over the batch in a fixed order
// (deterministic). dW1 = dH1^T X, dW2 = dH2^T H1, dW3 = dO^T H2, biases the column sums.
__global__ void mlp_grads(const float *X, const float *H1, const float *H2, const float *dH1,
                          const float *dH2, const float *dO, int B, float *G) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    float acc = 0.f;
    if (p < O_B1) {
        const int j = p / F, i = p % F;
        for (int b = 0; b < B; b++) acc = fmaf(dH1[int64_t(b) * H + j], X[int64_t(b) * F + i], acc);
    } else if (p < O_W2) {
        const int j = p - O_B1;
        for (int b = 0; b < B; b++) acc += dH1[int64_t(b) * H + j];
    } else if (p < O_B2) {
        const int j = (p - O_W2) / H, i = (p - O_W2) % H;
        for (int b = 0; b < B; b++) acc = fmaf(dH2[int64_t(b) * H + j], H1[int64_t(b) * H + i], acc);
    } else if (p < O_W3) {
        const int j = p - O_B2;
        for (int b = 0; b < B; b++) acc += dH2[int64_t(b) * H + j];
    } else if (p < O_B3) {
        const int j = p - O_W3;
        for (int b = 0; b < B; b++) acc = fmaf(dO[b], H2[int64_t(b) * H + j], acc);
    } else {
        for (int b = 0; b < B; b++) acc += dO[b];
    }
    G[p] = acc;
}

// Adam (Kingma & Ba) with bias correction, on the float32 masters.
__global__ void mlp_adam(float *P, const float *G, float *M, float *V, int n, float lr, float b1,
                         float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float g = G[p];
    const float m = b1 * M[p] + (1.f - b1) * g;
    const float v = b2 * V[p] + (1.f - b2) * g * g;
    M[p] = m;
    V[p] = v;
    P[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void mlp_predict_kernel(const float *P, const float *X, int n, float *out) {
    extern __shared__ float sw[];
    load_weights(P, sw);
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < n; b += warps) {
        float x[F];
#pragma unroll
        for (int i = 0; i < F; i++) x[i] = X[int64_t(b) * F + i];
        float h1a, h1b, h2a, h2b;
        const float o = forward(sw, x, lane, h1a, h1b, h2a, h2b);
        if (lane == 0) out[b] = o;
    }
}

// Inference layout used by the search kernel: bf16 W1, W2 and W3 in lane pairs, then float32 b1 [64],
// b2 [64], b3 [1], feature mean [12], feature 1/std [12]. A pair is the weights of hidden units l and
// l + 32 for one input, (W[l][i], W[l + 32][i]), stored at [i][l]: lane l reads both of its units'
// weights for input i in one 32-bit load.
__global__ void mlp_pack_kernel(const float *P, const float *mean, const float *inv_std,
                                unsigned char *dst) {
    __nv_bfloat16 *w = reinterpret_cast<__nv_bfloat16 *>(dst);
    float *b = reinterpret_cast<float *>(dst + size_t(H * F + H * H + H) * 2);
    for (int t = threadIdx.x; t < H * F; t += blockDim.x) {
        const int i = t / H, j = (t % H) / 2 + 32 * (t % 2);  // pair [i][l], half -> unit j
        w[t] = __float2bfloat16_rn(P[O_W1 + j * F + i]);
    }
    for (int t = threadIdx.x; t < H * H; t += blockDim.x) {
        const int i = t / H, j = (t % H) / 2 + 32 * (t % 2);
        w[H * F + t] = __float2bfloat16_rn(P[O_W2 + j * H + i]);
    }
    for (int t = threadIdx.x; t < H; t += blockDim.x) {
        w[H * F + H * H + t] = __float2bfloat16_rn(P[O_W3 + t / 2 + 32 * (t % 2)]);
        b[t] = P[O_B1 + t];
        b[H + t] = P[O_B2 + t];
    }
    if (threadIdx.x == 0) b[2 * H] = P[O_B3];
    for (int t = threadIdx.x; t < F; t += blockDim.x) {
        b[2 * H + 1 + t] = mean[t];
        b[2 * H + 1 + F + t] = inv_std[t];
    }
}

size_t scratch_floats(int B) { return size_t(B) * (4 * H + 1) + NPARAM + 4; }

}  // namespace hbm

extern "C" {

int64_t hnsw_b200_mlp_param_count(void) { return hbm::NPARAM; }

int64_t hnsw_b200_mlp_packed_bytes(void) {
    return int64_t(hbm::H * hbm::F + hbm::H * hbm::H + hbm::H) * 2 +
           int64_t(2 * hbm::H + 1 + 2 * hbm::F) * 4;
}

int64_t hnsw_b200_mlp_scratch_bytes(int32_t batch) {
    return batch < 1 ? 0 : int64_t(hbm::scratch_floats(batch) * sizeof(float));
}

int hnsw_b200_mlp_train_step(float *params, float *adam_m, float *adam_v, int64_t step, float lr,
                             const float *features, const float *targets, int32_t batch,
                             float *scratch, float *loss, void *stream) {
    using namespace hbm;
    if (!params || !adam_m || !adam_v || !features || !targets || !scratch || !loss || batch < 1 ||
        step < 1)
        return hb::fail(HNSW_B200_EINVAL, "mlp_train_step: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *H1 = scratch, *H2 = H1 + size_t(batch) * H, *dH1 = H2 + size_t(batch) * H;
    float *dH2 = dH1 + size_t(batch) * H, *dO = dH2 + size_t(batch) * H, *G = dO + batch;
    const int threads = 256;
    const int blocks = std::min(1184, (batch * 32 + threads - 1) / threads);
    cudaMemsetAsync(loss, 0, sizeof(float), s);
    mlp_fwd_bwd<<<blocks, threads, SMEM_FLOATS * sizeof(float), s>>>(params, features, targets,
                                                                       batch, H1, H2, dH1, dH2, dO, loss);
    mlp_grads<<<(NPARAM + 127) / 128, 128, 0, s>>>(features, H1, H2, dH1, dH2, dO, batch, G);
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    mlp_adam<<<(NPARAM + 255) / 256, 256, 0, s>>>(params, G, adam_m, adam_v, NPARAM, lr, b1, b2,
                                                  1e-8f, c1, c2);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("mlp train: ") + cudaGetErrorString(e));
    return 0;
}

// Gradients only (no update): G receives dLoss/dparams for the batch (for gradient checks).
int hnsw_b200_mlp_gradients(const float *params, const float *features, const float *targets,
                            int32_t batch, float *scratch, float *grads, float *loss, void *stream) {
    using namespace hbm;
    if (!params || !features || !targets || !scratch || !grads || !loss || batch < 1)
        return hb::fail(HNSW_B200_EINVAL, "mlp_gradients: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *H1 = scratch, *H2 = H1 + size_t(batch) * H, *dH1 = H2 + size_t(batch) * H;
    float *dH2 = dH1 + size_t(batch) * H, *dO = dH2 + size_t(batch) * H;
    const int threads = 256;
    const int blocks = std::min(1184, (batch * 32 + threads - 1) / threads);
    cudaMemsetAsync(loss, 0, sizeof(float), s);
    mlp_fwd_bwd<<<blocks, threads, SMEM_FLOATS * sizeof(float), s>>>(params, features, targets,
                                                                       batch, H1, H2, dH1, dH2, dO, loss);
    mlp_grads<<<(NPARAM + 127) / 128, 128, 0, s>>>(features, H1, H2, dH1, dH2, dO, batch, grads);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("mlp grads: ") + cudaGetErrorString(e));
    return 0;
}

int hnsw_b200_mlp_predict(const float *params, const float *features, int64_t n, float *out,
                          void *stream) {
    using namespace hbm;
    if (!params || !features || !out || n < 0) return hb::fail(HNSW_B200_EINVAL, "mlp_predict: bad argument");
    if (n == 0) return 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int threads = 256;
    const int blocks = int(std::min<int64_t>(2368, (n * 32 + threads - 1) / threads));
    mlp_predict_kernel<<<blocks, threads, SMEM_FLOATS * sizeof(float), s>>>(params, features, int(n), out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("mlp predict: ") + cudaGetErrorString(e));
    return 0;
}

int hnsw_b200_mlp_pack(const float *params, const float *mean, const float *inv_std, void *packed,
                       void *stream) {
    using namespace hbm;
    if (!params || !mean || !inv_std || !packed) return hb::fail(HNSW_B200_EINVAL, "mlp_pack: bad argument");
    mlp_pack_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        params, mean, inv_std, static_cast<unsigned char *>(packed));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("mlp pack: ") + cudaGetErrorString(e));
    return 0;
}

}  // extern "C"
