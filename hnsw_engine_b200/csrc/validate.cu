// On-device validation of a native graph (the checks of the reference's _validate_native,
// src/hnsw_engine/numba_engine.py:878-915, and of persistence.validate_state for links), run over
// the arrays already uploaded for searching instead of a host pass over the files.
//
// Every node and every upper-layer row is checked by its own thread. Each failed check sets one
// bit of a flag word; the host reports the first failed check in the order the host validator
// checks them, so the error is the one the host would raise. No check reads through a value it
// has not bounded first: link counts are clamped to the row width, link targets are range
// checked before they index levels, and upper-layer offsets are range checked before they index
// the row scratch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "hnsw_b200.h"

namespace hb {
int fail(int code, const std::string &msg);
}

namespace hbv {

__global__ void check_nodes(const int64_t *levels, const int32_t *count0, const int32_t *links0,
                            const int64_t *upper_offset, int64_t n, int64_t rows, int32_t stride0,
                            int32_t cap0, int32_t *cover, int32_t *row_layer, uint32_t *flags,
                            unsigned long long *top) {
    for (int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < n;
         u += int64_t(gridDim.x) * blockDim.x) {
        uint32_t f = 0;
        const int64_t lv = levels[u];
        if (lv < 0) f |= HNSW_B200_BAD_LEVEL;
        atomicMax(top, static_cast<unsigned long long>(lv < 0 ? 0 : lv));
        const int32_t c = count0[u];
        if (c < 0 || c > cap0) {
            f |= HNSW_B200_BAD_COUNT0;
        } else {
            const int32_t *row = links0 + u * stride0;
            for (int32_t j = 0; j < c; j++) {
                const int32_t t = row[j];
                if (t < 0 || t >= n) {
                    f |= HNSW_B200_BAD_LINK0;
                    break;
                }
            }
        }
        if (lv > 0) {
            const int64_t off = upper_offset[u];
            if (off < 0 || off > rows - lv) {
                f |= HNSW_B200_BAD_ROWS;
            } else {
                for (int64_t j = 0; j < lv; j++) {
                    atomicAdd(cover + off + j, 1);
                    row_layer[off + j] = int32_t(j + 1);
                }
            }
        }
        if (f) atomicOr(flags, f);
    }
}

__global__ void check_rows(const int64_t *levels, const int32_t *count_up, const int32_t *links_up,
                           int64_t n, int64_t rows, int32_t stride_up, int32_t cap_up,
                           const int32_t *cover, const int32_t *row_layer, uint32_t *flags) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows;
         r += int64_t(gridDim.x) * blockDim.x) {
        uint32_t f = 0;
        const bool tiled = cover[r] == 1;
        if (!tiled) f |= HNSW_B200_BAD_ROWS;
        const int32_t c = count_up[r];
        if (c < 0 || c > cap_up) {
            f |= HNSW_B200_BAD_COUNT_UP;
        } else {
            const int32_t *row = links_up + r * stride_up;
            for (int32_t j = 0; j < c; j++) {
                const int32_t t = row[j];
                if (t < 0 || t >= n) {
                    f |= HNSW_B200_BAD_LINK_UP;
                    break;
                }
                if (tiled && levels[t] < row_layer[r]) f |= HNSW_B200_BAD_LAYER;
            }
        }
        if (f) atomicOr(flags, f);
    }
}

}  // namespace hbv

extern "C" {

int64_t hnsw_b200_validate_scratch_bytes(int64_t rows) {
    return (rows > 0 ? rows : 0) * 2 * int64_t(sizeof(int32_t)) + 16;
}

int hnsw_b200_validate_graph(const hnsw_b200_graph_t *graph, const int64_t *levels, int32_t M,
                             void *scratch, uint32_t *flags_out, void *stream) {
    using namespace hbv;
    if (!graph || !levels || !scratch || !flags_out || M < 1)
        return hb::fail(HNSW_B200_EINVAL, "validate_graph: bad argument");
    const hnsw_b200_graph_t &g = *graph;
    if (g.n <= 0 || !g.links0 || !g.count0 || !g.upper_offset)
        return hb::fail(HNSW_B200_EINVAL, "validate_graph: the graph needs nodes and link arrays");
    if (g.rows > 0 && (!g.links_up || !g.count_up))
        return hb::fail(HNSW_B200_EINVAL, "validate_graph: upper rows need links_up and count_up");
    if (g.links0_stride < 2 * M || (g.rows > 0 && g.links_up_stride < M))
        return hb::fail(HNSW_B200_EINVAL, "validate_graph: row widths below the link capacities");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t rows = g.rows > 0 ? g.rows : 0;
    // Scratch layout: flags (u32) | pad | top (u64) | cover (rows i32) | row_layer (rows i32).
    unsigned char *base = static_cast<unsigned char *>(scratch);
    uint32_t *flags = reinterpret_cast<uint32_t *>(base);
    unsigned long long *top = reinterpret_cast<unsigned long long *>(base + 8);
    int32_t *cover = reinterpret_cast<int32_t *>(base + 16);
    int32_t *row_layer = cover + rows;
    cudaError_t e = cudaMemsetAsync(scratch, 0, size_t(hnsw_b200_validate_scratch_bytes(rows)), s);
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("validate: ") + cudaGetErrorString(e));
    const int threads = 256;
    const int nb = int(std::min<int64_t>(4096, (g.n + threads - 1) / threads));
    check_nodes<<<nb, threads, 0, s>>>(levels, g.count0, g.links0, g.upper_offset, g.n, rows,
                                       g.links0_stride, 2 * M, cover, row_layer, flags, top);
    if (rows > 0) {
        const int rb = int(std::min<int64_t>(4096, (rows + threads - 1) / threads));
        check_rows<<<rb, threads, 0, s>>>(levels, g.count_up, g.links_up, g.n, rows,
                                          g.links_up_stride, M, cover, row_layer, flags);
    }
    unsigned long long host[2] = {0, 0};
    e = cudaMemcpyAsync(host, base, 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("validate: ") + cudaGetErrorString(e));
    uint32_t f = uint32_t(host[0] & 0xffffffffu);
    // The entry point must be a node of the top layer, and max_level that layer.
    const unsigned long long t = host[1];
    int64_t ep_level = -1;
    if (g.entry_point >= 0 && g.entry_point < g.n) {
        e = cudaMemcpy(&ep_level, levels + g.entry_point, sizeof(int64_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return hb::fail(HNSW_B200_ECUDA, std::string("validate: ") + cudaGetErrorString(e));
    }
    if (int64_t(t) != int64_t(g.max_level) || ep_level != int64_t(t)) f |= HNSW_B200_BAD_ENTRY;
    *flags_out = f;
    return 0;
}

}  // extern "C"
