// Start order of a search batch: each query's cell -- its nearest pivot row -- and its predicted
// length, the start priority that hnsw_b200_search sorts into its first work list. The search
// kernel itself adds every finished query's expansions to the per-cell table (args->cells), so
// the prediction needs this one launch per batch and no host round trip.
//
// Nearest pivot: argmin over pivots of |p|^2 - 2 q.p (squared L2 less the query's own norm) in
// float32 -- exact for byte-valued data at d = 128, and a prediction input in any case, so the
// rounding is of no consequence; ties go to the lower pivot index. A block of 128 threads takes
// 16 queries; each thread holds two pivots of the current group of 256 and accumulates their dot
// products with all 16 queries. Queries and pivots arrive 32 dimensions at a time through shared
// memory: rows read whole (coalesced; the pivots as 16-byte pieces when the rows allow) and stored
// transposed, the queries read back as float4 broadcasts, the pivots one word per thread (the
// pivot tile's rows are padded by one word, so the transposing stores and the reads are free of
// bank conflicts). 10,000 queries make 625 blocks: one wave.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <string>

#include "hnsw_b200.h"

namespace hb {
int fail(int code, const std::string &msg);
}

namespace hbs {

constexpr int QT = 16;        // queries per block
constexpr int THREADS = 128;  // threads per block
constexpr int GROUP = 256;    // pivots per group: two per thread
constexpr int DC = 32;        // dimensions per staged chunk

__global__ void __launch_bounds__(THREADS) start_priority_kernel(
    const float *__restrict__ queries, int32_t nq, int32_t dim, const float *__restrict__ pivots,
    int32_t n_cells, const double *__restrict__ cost, const int32_t *__restrict__ ef, float scale,
    int32_t *__restrict__ cells, int32_t *__restrict__ priority, bool vec4) {
    __shared__ __align__(16) float qs[DC][QT];  // [dimension][query]
    __shared__ float ps[DC][GROUP + 1];         // [dimension][pivot of the group]
    __shared__ float wd[THREADS / 32][QT];
    __shared__ int wi[THREADS / 32][QT];
    __shared__ float best_d[QT];
    __shared__ int best_i[QT];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int q0 = blockIdx.x * QT;
    if (t < QT) {
        best_d[t] = FLT_MAX;
        best_i[t] = 0;
    }
    for (int g0 = 0; g0 < n_cells; g0 += GROUP) {
        const int pa = g0 + t, pb = g0 + THREADS + t;
        const bool la = pa < n_cells, lb = pb < n_cells;
        float acc_a[QT], acc_b[QT];
#pragma unroll
        for (int i = 0; i < QT; i++) {
            acc_a[i] = 0.f;
            acc_b[i] = 0.f;
        }
        float na = 0.f, nb = 0.f;  // |p|^2
        for (int d0 = 0; d0 < dim; d0 += DC) {
            __syncthreads();
            for (int e = t; e < QT * DC; e += THREADS) {  // stage 16 queries x 32 dimensions
                const int i = e / DC, d = e % DC;
                const int qi = q0 + i, dd = d0 + d;
                qs[d][i] = (qi < nq && dd < dim) ? queries[int64_t(qi) * dim + dd] : 0.f;
            }
            if (vec4 && d0 + DC <= dim) {
                // and 256 pivots x 32 dimensions, as 16-byte pieces: sixteen loads a thread in two
                // batches of eight (80 registers, so the 625 blocks of 10,000 queries stay one
                // wave), eight threads to a pivot's 128 bytes; piece k of pivot j lands in rows
                // 4k..4k+3 of the tile, banks 4k + c + j (mod 32), distinct across a warp
#pragma unroll 8
                for (int e = t; e < GROUP * DC / 4; e += THREADS) {
                    const int j = e / (DC / 4), k = e % (DC / 4);
                    const int pj = g0 + j;
                    const float4 v = pj < n_cells
                                         ? __ldg(reinterpret_cast<const float4 *>(
                                                     pivots + int64_t(pj) * dim + d0) + k)
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
                    ps[4 * k][j] = v.x;
                    ps[4 * k + 1][j] = v.y;
                    ps[4 * k + 2][j] = v.z;
                    ps[4 * k + 3][j] = v.w;
                }
            } else {
                for (int e = t; e < GROUP * DC; e += THREADS) {  // one word at a time
                    const int j = e / DC, d = e % DC;
                    const int pj = g0 + j, dd = d0 + d;
                    ps[d][j] = (pj < n_cells && dd < dim) ? __ldg(pivots + int64_t(pj) * dim + dd) : 0.f;
                }
            }
            __syncthreads();
            const int nd = min(DC, dim - d0);
            for (int d = 0; d < nd; d++) {
                const float va = ps[d][t];
                const float vb = ps[d][THREADS + t];
                na = fmaf(va, va, na);
                nb = fmaf(vb, vb, nb);
                const float4 *qv = reinterpret_cast<const float4 *>(qs[d]);
#pragma unroll
                for (int j = 0; j < QT / 4; j++) {
                    const float4 x = qv[j];
                    acc_a[4 * j] = fmaf(x.x, va, acc_a[4 * j]);
                    acc_a[4 * j + 1] = fmaf(x.y, va, acc_a[4 * j + 1]);
                    acc_a[4 * j + 2] = fmaf(x.z, va, acc_a[4 * j + 2]);
                    acc_a[4 * j + 3] = fmaf(x.w, va, acc_a[4 * j + 3]);
                    acc_b[4 * j] = fmaf(x.x, vb, acc_b[4 * j]);
                    acc_b[4 * j + 1] = fmaf(x.y, vb, acc_b[4 * j + 1]);
                    acc_b[4 * j + 2] = fmaf(x.z, vb, acc_b[4 * j + 2]);
                    acc_b[4 * j + 3] = fmaf(x.w, vb, acc_b[4 * j + 3]);
                }
            }
        }
        // argmin per query: the thread's two pivots, then the warp, then the block's warps
#pragma unroll
        for (int i = 0; i < QT; i++) {
            const float sa = la ? fmaf(-2.f, acc_a[i], na) : FLT_MAX;
            const float sb = lb ? fmaf(-2.f, acc_b[i], nb) : FLT_MAX;
            float v = sa;
            int id = la ? pa : INT32_MAX;
            if (sb < v) {  // pb > pa: equal scores keep pa
                v = sb;
                id = pb;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
                const int id2 = __shfl_xor_sync(0xffffffffu, id, o);
                if (v2 < v || (v2 == v && id2 < id)) {
                    v = v2;
                    id = id2;
                }
            }
            if (lane == 0) {
                wd[warp][i] = v;
                wi[warp][i] = id;
            }
        }
        __syncthreads();
        if (t < QT) {
            float v = best_d[t];
            int id = best_i[t];
            for (int w = 0; w < THREADS / 32; w++) {
                // lanes past n_cells carry (FLT_MAX, INT32_MAX) and never replace the entry
                if (wi[w][t] < n_cells && (wd[w][t] < v || (wd[w][t] == v && wi[w][t] < id))) {
                    v = wd[w][t];
                    id = wi[w][t];
                }
            }
            best_d[t] = v;
            best_i[t] = id;
        }
    }
    __syncthreads();
    if (t < QT && q0 + t < nq) {
        const int q = q0 + t, c = best_i[t];
        // expansions per unit of ef: plain searches' mean where they reached the cell, else the
        // stopped searches' (0 for a cell nobody reached yet)
        const double plain_n = cost[2 * int64_t(n_cells) + c];
        const double ratio = plain_n > 0.0
                                 ? cost[c] / plain_n
                                 : cost[int64_t(n_cells) + c] / fmax(1.0, cost[3 * int64_t(n_cells) + c]);
        const double key = fmin(65535.0, ratio * double(ef[q]) * double(scale));
        cells[q] = c;
        priority[q] = int32_t(key);
    }
}

}  // namespace hbs

extern "C" int hnsw_b200_start_priority(const float *queries, int64_t nq, int32_t dim,
                                        const float *pivots, int32_t n_cells, const double *cost,
                                        const int32_t *ef, float scale, int32_t *cells,
                                        int32_t *priority, void *stream) {
    if (nq < 0 || nq > INT32_MAX || dim < 1 || n_cells < 1 || !(scale >= 0.f))
        return hb::fail(HNSW_B200_EINVAL, "start_priority: bad sizes");
    if (nq == 0) return HNSW_B200_OK;
    if (!queries || !pivots || !cost || !ef || !cells || !priority)
        return hb::fail(HNSW_B200_EINVAL, "start_priority: null pointer");
    const int blocks = int((nq + hbs::QT - 1) / hbs::QT);
    hbs::start_priority_kernel<<<blocks, hbs::THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        queries, int32_t(nq), dim, pivots, n_cells, cost, ef, scale, cells, priority,
        (dim & 3) == 0 && (reinterpret_cast<uintptr_t>(pivots) & 15) == 0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("start_priority: ") + cudaGetErrorString(e));
    return HNSW_B200_OK;
}
