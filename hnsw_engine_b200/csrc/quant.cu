// Scalar quantizer fit and encode on the GPU (the reference's ScalarQuantizer.fit / encode,
// src/hnsw_engine/quantization.py:37-59), over the float32 rows already resident for searching.
//
// fit needs per-dimension minima and maxima and whether every value is an integer; encode is
// code = clip(rint((double(x) - offset[j]) / step), 0, 255) in float64 -- the reference's NumPy
// arithmetic: the float32 value widened exactly, one correctly rounded subtraction and division,
// round half to even, clip -- so the codes are the reference's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "hnsw_b200.h"

namespace hb {
int fail(int code, const std::string &msg);
}

namespace hbq {

// Order-preserving keys of float32 values: ascending floats -> ascending unsigned keys.
__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// One thread per dimension column slice: block b reduces rows [b * rows_per, ...) of every
// dimension (threads stride over dimensions), then one atomic per dimension and block.
__global__ void column_stats(const float *x, int64_t n, int dim, int64_t rows_per, uint32_t *kmin,
                             uint32_t *kmax, int32_t *nonint) {
    const int64_t r0 = int64_t(blockIdx.x) * rows_per;
    const int64_t r1 = min(n, r0 + rows_per);
    int bad = 0;
    for (int j = threadIdx.x; j < dim; j += blockDim.x) {
        uint32_t lo = 0xffffffffu, hi = 0u;
        for (int64_t r = r0; r < r1; r++) {
            const float v = x[r * dim + j];
            const uint32_t k = fkey(v);
            lo = min(lo, k);
            hi = max(hi, k);
            bad |= v != rintf(v);
        }
        if (r0 < r1) {
            atomicMin(kmin + j, lo);
            atomicMax(kmax + j, hi);
        }
    }
    if (bad) atomicOr(nonint, 1);
}

__global__ void encode_rows(const float *x, int64_t total, int dim, const double *offset, double step,
                            uint8_t *codes) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int j = int(i % dim);
        const double c = rint((double(x[i]) - offset[j]) / step);
        codes[i] = uint8_t(c < 0.0 ? 0.0 : (c > 255.0 ? 255.0 : c));
    }
}

__device__ __forceinline__ float funkey(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void unkey(const uint32_t *kmin, const uint32_t *kmax, int dim, double *lo, double *hi) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < dim; j += gridDim.x * blockDim.x) {
        lo[j] = double(funkey(kmin[j]));
        hi[j] = double(funkey(kmax[j]));
    }
}

}  // namespace hbq

extern "C" {

int64_t hnsw_b200_quant_scratch_bytes(int32_t dim) { return int64_t(dim > 0 ? dim : 0) * 8 + 16; }

int hnsw_b200_quant_stats(const float *vectors, int64_t n, int32_t dim, double *lo, double *hi,
                          int32_t *integer_valued, void *scratch, void *stream) {
    using namespace hbq;
    if (!vectors || !lo || !hi || !integer_valued || !scratch || n <= 0 || dim <= 0)
        return hb::fail(HNSW_B200_EINVAL, "quant_stats: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t *kmin = static_cast<uint32_t *>(scratch);
    uint32_t *kmax = kmin + dim;
    int32_t *nonint = reinterpret_cast<int32_t *>(kmax + dim);
    cudaError_t e = cudaMemsetAsync(kmin, 0xff, size_t(dim) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(kmax, 0, size_t(dim) * 4 + 16, s);
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("quant_stats: ") + cudaGetErrorString(e));
    const int64_t blocks = std::min<int64_t>(4096, n);
    const int64_t rows_per = (n + blocks - 1) / blocks;
    const int64_t nb = (n + rows_per - 1) / rows_per;
    const int threads = std::min(256, ((dim + 31) / 32) * 32);
    column_stats<<<int(nb), threads, 0, s>>>(vectors, n, dim, rows_per, kmin, kmax, nonint);
    unkey<<<std::max(1, (dim + 255) / 256), 256, 0, s>>>(kmin, kmax, dim, lo, hi);
    int32_t h = 0;
    e = cudaMemcpyAsync(&h, nonint, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("quant_stats: ") + cudaGetErrorString(e));
    *integer_valued = h ? 0 : 1;
    return 0;
}

int hnsw_b200_quant_encode(const float *vectors, int64_t n, int32_t dim, const double *offset,
                           double step, uint8_t *codes, void *stream) {
    using namespace hbq;
    if (!vectors || !offset || !codes || n <= 0 || dim <= 0 || !(step > 0.0))
        return hb::fail(HNSW_B200_EINVAL, "quant_encode: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t total = n * dim;
    const int blocks = int(std::min<int64_t>(148 * 16, (total + 255) / 256));
    encode_rows<<<blocks, 256, 0, s>>>(vectors, total, dim, offset, step, codes);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("quant_encode: ") + cudaGetErrorString(e));
    return 0;
}

}  // extern "C"
