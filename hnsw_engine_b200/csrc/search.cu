// Batched HNSW search on B200 (sm_100a): one warp per query, persistent grid fed by an atomic
// work queue.
//
// Semantics are those of the reference's compiled search (anamankev/hnsw-engine):
//   _search_batch            src/hnsw_engine/numba_engine.py:422-503  -> search_kernel
//   _search_layer            numba_engine.py:98-148                    -> layer_search
//   _search_layer0_filtered  numba_engine.py:151-198                   -> layer0_filtered
//   _distance                numba_engine.py:57-70                     -> dist_seq_f64 / dists_exact_f32
//   _rerank_batch            numba_engine.py:506-530                   -> rerank_epilogue
// and the canonical rules of the reference project's own docs/DESIGN.md, section 5 (rules 4, 5,
// 9): candidates pop in ascending (distance, id); a neighbour is admitted iff the results hold
// fewer than ef entries or its distance is strictly below the running worst, neighbours taken in
// stored link order; the worst result (maximum (distance, id)) is evicted.
//
// Data structures (per query, one warp):
//  * results R: a sorted (distance, id) array in shared memory with an "expanded" bit per entry.
//    In an unfiltered layer every unexpanded result is a pending candidate, and every other pending
//    candidate ties the worst distance (it was evicted as the maximum while the worst stayed the
//    same), so the reference's unbounded candidate heap reduces to R plus a stack of tied ids
//    (`ties`, popped smallest id first). Candidates farther than the worst are dropped: once the
//    results are full the worst never grows, so the reference would stop on them.
//  * filtered layer 0 keeps candidates explicitly (disallowed nodes are candidates but never
//    results): a descending sorted array S in shared memory plus an unsorted global spill G whose
//    entries all compare above every entry of S; S is refilled with the smallest entries of G.
//  * visited: an exact open-addressing hash of node ids per warp slot in global memory (L2
//    resident), cleared per layer, as the reference's epoch-stamped array is per layer.
// Any capacity overflow sets a per-query status bit; the host re-runs those queries with larger
// scratch, so results are always exact. Nothing traps and every loop is bounded.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "hnsw_b200.h"

namespace hb {

constexpr unsigned FULL = 0xffffffffu;
constexpr int32_t EXP_BIT = int32_t(0x80000000u);
constexpr int32_t ID_MASK = 0x7fffffff;
constexpr int WPB = 4;  // warps per block

// Minimum resident blocks per SM requested from the compiler (caps registers per thread), per
// arithmetic mode, and rows in flight per lane in the distance loops. Tuned on B200.
#ifndef HB_MINB_F64
#define HB_MINB_F64 5  // 6 blocks spill at 80 registers: t1m ef = 64 4.09 against 3.71 ms at 5
#endif
#ifndef HB_MINB_EXACT
#define HB_MINB_EXACT 4
#endif
#ifndef HB_MINB_BYTES
#define HB_MINB_BYTES 5
#endif
#ifndef HB_MINB_BYTES_FILT
#define HB_MINB_BYTES_FILT 5
#endif
#ifndef HB_NB_EXACT
#define HB_NB_EXACT 4
#endif
#ifndef HB_NB_BYTES
#define HB_NB_BYTES 8
#endif
// Layer 0: admit a chunk's neighbours together (exactly the sequential outcome) instead of one by one.
#ifndef HB_BATCH_ADMIT
#define HB_BATCH_ADMIT 1
#endif
// Byte rows of at most 128 bytes: one lane per neighbour, row loads issued before the visited marks.
#ifndef HB_LANE_ROWS
#define HB_LANE_ROWS 1
#endif
// 128-byte rows gathered a line per group of eight lanes (mark_score_group_rows) instead of a row
// per lane: an eighth of the L1 wavefronts for the same lines. 1M mixture, 10K queries, identical
// results: ef = 64 1.39 -> 1.26 ms, ef = 192 3.24 -> 2.95 ms, learned stop 3.34 -> 3.05 ms.
#ifndef HB_GROUP_ROWS
#define HB_GROUP_ROWS 1
#endif
// Filtered searches gather rows before the visited marks only above this allowed share. With the
// group gather, gathering at every share measured mixed on the 1M mixture (10K queries, one call):
// Bernoulli p = 0.03 ef = 64 49.4 -> 43.8 ms and p = 0.01 ef = 192 657 -> 636 ms, but p = 0.03
// ef = 192 160 -> 167 ms and p = 0.01 ef = 64 165 -> 172 ms; the 5% cut stays.
#ifndef HB_LANE_ROWS_MIN_P
#define HB_LANE_ROWS_MIN_P 0.05
#endif
// Byte codes in float64 sums: read four codes a load (dim a multiple of 4). Identical results;
// int8 codes of the 1M x 100 cosine graph with the float64 rerank at ef = 128: 6.31 -> 6.16 ms.
#ifndef HB_CODE_WORDS
#define HB_CODE_WORDS 1
#endif
// Batched admission (unfiltered and filtered): rank a candidate in R (and in the filtered
// candidates S) by a binary search whose step count depends on the array's length alone, so the
// lanes never diverge in it (uniform_prefix). Identical results; 1M mixture, 10K queries: ef = 192
// 2.927 -> 2.907 ms, learned stop 3.04 -> 3.00 ms.
#ifndef HB_UNIFORM_RANK
#define HB_UNIFORM_RANK 1
#endif
// Float64 rows: prefetch a row's lines into L1 before its sequential sum (prefetch_row_l1).
// Identical results; t1m (1M x 100 cosine, 10K queries) ef = 256 10.81 -> 9.59 ms, its int8 codes
// with the float64 rerank at ef = 128 6.72 -> 6.47 ms, the 1M mixture in float64 at ef = 192
// 6.76 -> 6.45 ms. Loading the row into registers in batches of 4 or 8 pieces instead spilled
// 0.3-3 KB a thread (the float64 kernels already hold 96 registers).
#ifndef HB_F64_PREFETCH
#define HB_F64_PREFETCH 1
#endif
// Batched admission: one pass over the chunk's candidates builds each lane's "below me" masks
// (3.5% faster than counting over the admitted set in a second pass: 3.45 -> 3.33 ms at ef = 192 on
// the 1M mixture, identical results).
#ifndef HB_ADMIT_MASKS
#define HB_ADMIT_MASKS 1
#endif
// Filtered layer 0: admit a chunk's neighbours together (exactly the one-by-one outcome).
#ifndef HB_BATCH_ADMIT_FILT
#define HB_BATCH_ADMIT_FILT 1
#endif
#ifdef HB_PROFILE
__device__ unsigned long long hb_prof[8];
#define HB_PROF_DECL unsigned long long hb_t = clock64();
#define HB_PROF(i)                           \
    do {                                     \
        unsigned long long hb_n = clock64(); \
        C.prof[i] += hb_n - hb_t;            \
        hb_t = hb_n;                         \
    } while (0)
#else
#define HB_PROF_DECL
#define HB_PROF(i) \
    do {           \
    } while (0)
#endif

// Kernel configurations among which the autotuner picks, for the byte kernels (the other modes
// build configuration 0 only): the resident blocks per SM requested from the compiler (which caps
// the registers per thread), the gathered rows of one lane per neighbour held in registers or
// staged in shared memory by cp.async, and the unfiltered layer-0 visited set as the per-slot
// bitmap or a per-slot open-addressing hash. Every configuration gives the same results.
constexpr int N_CONFIGS = 4;
__host__ __device__ constexpr int cfg_blocks(int c) { return c == 1 ? 4 : 5; }
__host__ __device__ constexpr bool cfg_stage(int c) { return c == 2; }
__host__ __device__ constexpr bool cfg_hash(int c) { return c == 3; }
inline const char *cfg_name(int c) {
    return c == 0 ? "bitmap, rows in registers, 5 blocks/SM"
                  : c == 1 ? "bitmap, rows in registers, 4 blocks/SM"
                           : c == 2 ? "bitmap, rows staged by cp.async, 5 blocks/SM"
                                    : "hash, rows in registers, 5 blocks/SM";
}
// Configurations built for a mode (byte kernels: all; the others: configuration 0).
__host__ __device__ constexpr int configs_of(int mode) { return mode == 2 ? N_CONFIGS : 1; }

// Resident blocks per SM requested for a kernel. Filtered byte searches: 5 blocks (96 registers)
// against 6 (80 registers, spilling 184 bytes) measured 4.18 against 4.72 ms at Bernoulli p = 0.5
// and 17.2 against 18.9 ms at p = 0.1 on the 1M mixture (float32 candidates).
template <int MODE, bool FILT, int CFG>
constexpr int min_blocks() {
    if (MODE == 2) return CFG == 0 ? (FILT ? HB_MINB_BYTES_FILT : HB_MINB_BYTES) : cfg_blocks(CFG);
    return MODE == 1 ? HB_MINB_EXACT : HB_MINB_F64;
}

enum : int32_t { ST_VISITED = 1, ST_TIES = 2, ST_SPILL = 4 };
enum : int { MODE_F64 = 0, MODE_EXACT = 1, MODE_BYTES = 2 };

struct SearchParams {
    const float *vectors;
    const uint8_t *codes;
    const uint8_t *rows8;  // byte mode: the uint8 rows searched
    // fused rerank: the vectors' uint8 copy (integer vectors in [0, 255]; L2 or inner product,
    // dim a multiple of 16 up to 128), or NULL
    const uint8_t *rerank_rows8;
    const int32_t *links0;
    const int32_t *count0;
    const int64_t *upper_offset;
    const int32_t *links_up;
    const int32_t *count_up;
    int64_t n;
    const int32_t *node_ids;  // original id of each internal node (NULL: internal = original)
    int32_t dim, links0_stride, links_up_stride, metric;
    int64_t entry_point;
    int32_t max_level;
    // batch
    const void *queries;
    int32_t queries_f64;
    const int32_t *qlist;  // work item -> query row (NULL: identity)
    int32_t n_work;
    const int32_t *cells;  // per-cell cost learning (NULL: off)
    double *cell_cost;     // (4, n_cells): plain sums, stopped sums, plain counts, stopped counts
    int32_t n_cells;
    int32_t k, k_search;
    const int32_t *ef;
    int32_t ef_cap;
    const uint32_t *allowed;
    const float *rerank_queries;
    int64_t *out_ids;
    double *out_dists;
    int64_t *out_ctr;
    int32_t *status;
    int32_t *n_failed;
    int32_t *queue;
    // scratch (per warp slot)
    uint32_t *vbits;      // layer-0 visited bitmap, one bit per node, all zero between queries
    int64_t vbits_stride; // words per slot
    int32_t *vlist;       // ids marked in the bitmap (to clear them), vlist_cap per slot
    int32_t vlist_cap;
    int32_t *vis;
    int64_t vis_stride;
    int32_t vis_log2, vis_up_log2;
    int32_t *ties;
    int32_t tie_cap;
    double *spill_d;
    int32_t *spill_i;       // original ids of spilled candidates
    int32_t *spill_p;       // their internal ids (graphs in an internal order; else spill_i)
    int32_t spill_cap;
    int32_t s_cap;
    // learned early termination (layer 0, unfiltered): features every STOP_EVERY expansions
    const void *stop_mlp;   // packed network (see mlp_smem_bytes), or NULL
    float stop_threshold;   // stop once the predicted further recall@k hits fall below it,
    float stop_slope;       // plus stop_slope per 64 layer-0 expansions beyond stop_slope_from
    int32_t stop_slope_from;
    float *trace_feat;      // (n_queries, trace_cap, STOP_FEATURES) or NULL
    double *trace_dk;       // (n_queries, trace_cap, trace_k): first results' distances per checkpoint
    int32_t *trace_count;   // (n_queries,) checkpoints recorded
    int32_t *trace_hops;    // (n_queries,) layer-0 expansions of the whole search
    int32_t trace_cap;
    int32_t trace_k;        // distances recorded per checkpoint (min(k, 16))
    int32_t lane_rows;      // byte rows may use mark_score_lane_rows (see the host's choice)
};

constexpr int STOP_EVERY = 16;
constexpr int STOP_FEATURES = 12;
constexpr int STOP_HIDDEN = 64;
// Packed network in device memory: bf16 W1 (12 x 32 pairs), W2 (64 x 32 pairs), W3 (32 pairs), then
// float32 b1 (64), b2 (64), b3 (1), feature mean (12), feature 1/std (12). Pair [i][l] holds the
// weights of hidden units l and l + 32 for input i, so lane l reads both in one 32-bit load
// without bank conflicts; features are standardised in the kernel.
constexpr int MLP_W1 = STOP_FEATURES * STOP_HIDDEN;
constexpr int MLP_W2 = STOP_HIDDEN * STOP_HIDDEN;
constexpr int MLP_W3 = STOP_HIDDEN;
constexpr int MLP_BF16 = MLP_W1 + MLP_W2 + MLP_W3;           // 4928 bf16 values
constexpr int MLP_F32 = STOP_HIDDEN + STOP_HIDDEN + 1 + 2 * STOP_FEATURES;  // 153 floats
constexpr size_t MLP_BYTES = size_t(MLP_BF16) * 2 + size_t(MLP_F32) * 4;

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

// Result slots per warp: ef_cap entries, plus room for a whole chunk of 32 admissions merged in
// before the excess is evicted (batched admission), plus one for sequential insertion.
__host__ __device__ inline int result_slots(int ef_cap) { return ef_cap + 33; }

// Shared memory of one warp: results, query (f64, f32 and bytes), filtered candidates, rerank top-k.
// two_ids: the graph is stored in an internal node order, so filtered results and candidates keep
// internal ids next to the original ones (otherwise, and always for unfiltered searches, whose
// results hold internal ids only, the two are the same array).
__host__ __device__ inline size_t warp_smem_bytes(int ef_cap, int dim, bool filtered, int s_cap,
                                                  int k_rerank, bool two_ids, int stage = 0) {
    size_t b = al16(size_t(stage)) + al16(size_t(result_slots(ef_cap)) * 8) +
               (two_ids && filtered ? 2 : 1) * al16(size_t(result_slots(ef_cap)) * 4) +
               al16(size_t(dim) * 8) +
               al16(size_t(dim) * 4) + al16(size_t(dim));
    if (filtered) b += al16(size_t(s_cap + 1) * 8) + (two_ids ? 2 : 1) * al16(size_t(s_cap + 1) * 4);
    if (k_rerank > 0) b += al16(size_t(k_rerank + 1) * 8) + al16(size_t(k_rerank + 1) * 4);
    return b;
}

// Shared-memory staging of gathered byte rows (bytes per warp: one row per lane), or 0.
__host__ __device__ inline int stage_bytes(int mode, int cfg, int lane_rows, int dim) {
    return (cfg_stage(cfg) && mode == 2 && lane_rows && (dim & 15) == 0 && dim <= 128) ? 32 * dim : 0;
}

// D: the type of the result and candidate distances (Rd, Sd, spd). Byte searches use float --
// their distances are integers of magnitude at most 128 * 255^2 < 2^24, exact in float32, so order
// and ties are unchanged -- halving the lists' shuffles and memory traffic and keeping their
// compares off the FP64 pipe. Every other search uses double.
template <typename D>
struct CtxT {
    using dist_t = D;
    int lane;
    D *Rd;
    int32_t *Ri;  // original id of each result (ordering, output), with the expanded bit
    int32_t *Rp;  // internal id of each result (memory accesses)
    double *qd;
    float *qf;
    uint32_t *q4;  // query bytes, four per word (byte mode)
    D *Sd;
    int32_t *Si;  // candidates: original ids
    int32_t *Sp;  // candidates: internal ids (the same array as Si unless the order differs)
    double *Ad;
    int32_t *Ai;
    int32_t *vis;
    uint32_t *vbits;
    int32_t *vlist;
    int32_t vlist_n;  // ids appended to vlist (may exceed the capacity: then clear everything)
    int32_t *ties;
    D *spd;
    int32_t *spi;
    int32_t *spp;
    long long ndist, nhops;  // uniform across the warp
    int32_t status;          // uniform across the warp
    int32_t q;               // query row
    bool lane_rows;          // byte rows fit one lane (dim a multiple of 16, at most 128)
    unsigned char *stage;    // this warp's row staging (one row per lane), or NULL
#ifdef HB_PROFILE
    unsigned long long prof[8];  // cycles per phase of this warp's current query
#endif
    float qfeat;             // log1p(|q|^2), a stop feature
    const __nv_bfloat16 *mlp_w;  // block shared memory copy of the network (or NULL)
    const float *mlp_b;
};
using Ctx = CtxT<double>;  // filtered searches and the float64 modes

// Node arrays may be stored in any order (internal ids, chosen for memory locality); results,
// and ties between equal distances, use the original ids. Unfiltered result lists hold internal
// ids and look the original ones up only for equal distances and at output. Sentinel ids outside
// [0, n) map to themselves.
__device__ __forceinline__ int32_t orig_id(const SearchParams &P, int32_t i) {
    return (P.node_ids != nullptr && i >= 0 && i < P.n) ? __ldg(P.node_ids + i) : i;
}

// (distance, id) order of two entries whose ids are comparable as they are.
template <typename T>
__device__ __forceinline__ bool pair_lt_raw(T da, int32_t ia, T db, int32_t ib) {
    return da < db || (da == db && ia < ib);
}

// (distance, original id) order of two entries held by internal id: the id lookups run only for
// equal distances, so the unfiltered result list carries internal ids alone.
template <typename T>
__device__ __forceinline__ bool pair_lt_int(const SearchParams &P, T da, int32_t ia, T db,
                                            int32_t ib) {
    if (da != db) return da < db;
    return orig_id(P, ia) < orig_id(P, ib);
}


// ---------------------------------------------------------------------------------------- sorted
// Entries of the ascending array [0, m) strictly below (d, id).
template <typename T>
__device__ __forceinline__ int count_below(const T *Ad, const int32_t *Ai, int m, T d,
                                           int32_t id, int lane) {
    int c = 0;
    for (int i = lane; i < m; i += 32) c += pair_lt_raw(Ad[i], Ai[i] & ID_MASK, d, id);
    return __reduce_add_sync(FULL, c);
}

// Same as count_below for a sorted ascending array, by a two-level warp search: 32 splitters, then
// the chunk that holds the boundary (exact for m <= 1024; falls back to the linear count beyond).
template <typename T>
__device__ __forceinline__ int sorted_rank(const T *Ad, const int32_t *Ai, int m, T d,
                                           int32_t id, int lane) {
    if (m > 1024) return count_below(Ad, Ai, m, d, id, lane);
    const int step = (m + 31) >> 5;  // entries per chunk
    const int s = lane * step;
    const bool below = s < m && pair_lt_raw(Ad[s], Ai[s] & ID_MASK, d, id);
    const uint32_t b = __ballot_sync(FULL, below);  // chunks starting below (d, id): a prefix
    const int chunks = __popc(b);
    if (chunks == 0) return 0;
    const int base = (chunks - 1) * step;  // the last chunk starting below holds the boundary
    const int i = base + lane;
    const bool in = lane < step && i < m && pair_lt_raw(Ad[i], Ai[i] & ID_MASK, d, id);
    return base + __popc(__ballot_sync(FULL, in));
}

// sorted_rank over entries held by internal ids (ordered by distance, then original id).
template <typename T>
__device__ __forceinline__ int sorted_rank_int(const SearchParams &P, const T *Ad,
                                               const int32_t *Ai, int m, T d, int32_t id,
                                               int lane) {
    if (m > 1024) {
        int c = 0;
        for (int i = lane; i < m; i += 32) c += pair_lt_int(P, Ad[i], Ai[i] & ID_MASK, d, id);
        return __reduce_add_sync(FULL, c);
    }
    const int step = (m + 31) >> 5;
    const int s = lane * step;
    const bool below = s < m && pair_lt_int(P, Ad[s], Ai[s] & ID_MASK, d, id);
    const uint32_t b = __ballot_sync(FULL, below);
    const int chunks = __popc(b);
    if (chunks == 0) return 0;
    const int base = (chunks - 1) * step;
    const int i = base + lane;
    const bool in = lane < step && i < m && pair_lt_int(P, Ad[i], Ai[i] & ID_MASK, d, id);
    return base + __popc(__ballot_sync(FULL, in));
}

// Entries of the descending array [0, m) strictly above (d, id).
template <typename T>
__device__ __forceinline__ int count_above(const T *Ad, const int32_t *Ai, int m, T d,
                                           int32_t id, int lane) {
    int c = 0;
    for (int i = lane; i < m; i += 32) c += pair_lt_raw(d, id, Ad[i], Ai[i]);
    return __reduce_add_sync(FULL, c);
}

// Move [pos, m) to [pos + 1, m + 1), highest chunk first (Ap: an optional third array).
template <typename T>
__device__ __forceinline__ void shift_up(T *Ad, int32_t *Ai, int pos, int m, int lane,
                                         int32_t *Ap = nullptr) {
    for (int top = m - 1; top >= pos; top -= 32) {
        int i = top - lane;
        bool act = i >= pos;
        T d = T(0);
        int32_t id = 0, ip = 0;
        if (act) {
            d = Ad[i];
            id = Ai[i];
            if (Ap) ip = Ap[i];
        }
        __syncwarp();
        if (act) {
            Ad[i + 1] = d;
            Ai[i + 1] = id;
            if (Ap) Ap[i + 1] = ip;
        }
        __syncwarp();
    }
}

// Move [pos + 1, m) to [pos, m - 1), lowest chunk first (Ap: an optional third array).
template <typename T>
__device__ __forceinline__ void shift_down(T *Ad, int32_t *Ai, int pos, int m, int lane,
                                           int32_t *Ap = nullptr) {
    for (int base = pos; base < m - 1; base += 32) {
        int i = base + lane;
        bool act = i < m - 1;
        T d = T(0);
        int32_t id = 0, ip = 0;
        if (act) {
            d = Ad[i + 1];
            id = Ai[i + 1];
            if (Ap) ip = Ap[i + 1];
        }
        __syncwarp();
        if (act) {
            Ad[i] = d;
            Ai[i] = id;
            if (Ap) Ap[i] = ip;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------- visited
// Length of the prefix of [0, m) on which pred holds (pred true on a prefix, false after), by a
// binary search whose step count depends on m alone: the lanes of a warp never diverge in it.
template <class F>
__device__ __forceinline__ int uniform_prefix(int m, F pred) {
    int a = 0;  // the answer stays within [a, a + n]
    for (int n = m; n > 1;) {
        const int half = n >> 1;
        a = pred(a + half - 1) ? a + half : a;
        n -= half;
    }
    if (m > 0 && pred(a)) a++;
    return a;
}

__device__ __forceinline__ void vis_clear(int32_t *tab, int log2, int lane) {
    int4 *t4 = reinterpret_cast<int4 *>(tab);
    const int n4 = (1 << log2) >> 2;
    for (int i = lane; i < n4; i += 32) t4[i] = make_int4(0, 0, 0, 0);
    __syncwarp();
}

// 1: inserted (was unvisited); 0: already present; -1: table full.
__device__ __forceinline__ int vis_insert(int32_t *tab, int log2, int32_t id) {
    const uint32_t mask = (1u << log2) - 1u;
    uint32_t h = (uint32_t(id) * 2654435761u) >> (32 - log2);
    const int32_t key = id + 1;
    for (uint32_t p = 0; p <= mask; p++) {
        int32_t old = atomicCAS(tab + h, 0, key);
        if (old == 0) return 1;
        if (old == key) return 0;
        h = (h + 1u) & mask;
    }
    return -1;
}

__device__ __forceinline__ bool is_allowed(const uint32_t *bits, int32_t e) {
    return (__ldg(bits + (e >> 5)) >> (e & 31)) & 1u;
}

// -------------------------------------------------------------------------------------- distances
// Float64, strictly sequential over the dimensions with separate multiply and add: the exact
// arithmetic of numba_engine._distance (:57-70) for float32 or uint8 rows and a float64 query.
// Ask the L1 for every line of a row before its sequential sum reads it: the lines arrive in one
// memory round trip instead of one round trip per load of the sum's loop, with no registers held.
__device__ __forceinline__ void prefetch_row_l1(const void *row, int bytes) {
    const char *b = static_cast<const char *>(row);
    for (int o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L1 [%0];" ::"l"(b + o));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(b + bytes - 1));
}

template <bool U8>
__device__ __forceinline__ double dist_seq_f64(const SearchParams &P, int64_t e, const double *q) {
    const int dim = P.dim;
    double acc = 0.0;
#if HB_F64_PREFETCH
    if (!U8) prefetch_row_l1(P.vectors + e * dim, dim * 4);
    else prefetch_row_l1(P.codes + e * dim, dim);
#endif
    if (!U8) {
        const float *x = P.vectors + e * dim;
        if ((dim & 3) == 0) {
            const float4 *x4 = reinterpret_cast<const float4 *>(x);
            if (P.metric == HNSW_B200_L2) {
                for (int i = 0; i < dim; i += 4) {
                    float4 v = __ldg(x4 + (i >> 2));
                    double t;
                    t = __dsub_rn((double)v.x, q[i]);
                    acc = __dadd_rn(acc, __dmul_rn(t, t));
                    t = __dsub_rn((double)v.y, q[i + 1]);
                    acc = __dadd_rn(acc, __dmul_rn(t, t));
                    t = __dsub_rn((double)v.z, q[i + 2]);
                    acc = __dadd_rn(acc, __dmul_rn(t, t));
                    t = __dsub_rn((double)v.w, q[i + 3]);
                    acc = __dadd_rn(acc, __dmul_rn(t, t));
                }
                return acc;
            }
            for (int i = 0; i < dim; i += 4) {
                float4 v = __ldg(x4 + (i >> 2));
                acc = __dadd_rn(acc, __dmul_rn((double)v.x, q[i]));
                acc = __dadd_rn(acc, __dmul_rn((double)v.y, q[i + 1]));
                acc = __dadd_rn(acc, __dmul_rn((double)v.z, q[i + 2]));
                acc = __dadd_rn(acc, __dmul_rn((double)v.w, q[i + 3]));
            }
        } else {
            if (P.metric == HNSW_B200_L2) {
                for (int i = 0; i < dim; i++) {
                    double t = __dsub_rn((double)__ldg(x + i), q[i]);
                    acc = __dadd_rn(acc, __dmul_rn(t, t));
                }
                return acc;
            }
            for (int i = 0; i < dim; i++) acc = __dadd_rn(acc, __dmul_rn((double)__ldg(x + i), q[i]));
        }
    } else {
        const uint8_t *x = P.codes + e * dim;
#if HB_CODE_WORDS
        if ((dim & 3) == 0) {  // four codes a load (rows start on 4-byte boundaries), same order
            const uint32_t *x4 = reinterpret_cast<const uint32_t *>(x);
            const bool l2 = P.metric == HNSW_B200_L2;
            for (int i = 0; i < dim; i += 4) {
                const uint32_t w = __ldg(x4 + (i >> 2));
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const double c = double((w >> (8 * u)) & 0xffu);
                    if (l2) {
                        const double t = __dsub_rn(c, q[i + u]);
                        acc = __dadd_rn(acc, __dmul_rn(t, t));
                    } else {
                        acc = __dadd_rn(acc, __dmul_rn(c, q[i + u]));
                    }
                }
            }
            if (l2) return acc;
            return P.metric == HNSW_B200_IP ? -acc : __dsub_rn(1.0, acc);
        }
#endif
        if (P.metric == HNSW_B200_L2) {
            for (int i = 0; i < dim; i++) {
                double t = __dsub_rn((double)__ldg(x + i), q[i]);
                acc = __dadd_rn(acc, __dmul_rn(t, t));
            }
            return acc;
        }
        for (int i = 0; i < dim; i++) acc = __dadd_rn(acc, __dmul_rn((double)__ldg(x + i), q[i]));
    }
    return P.metric == HNSW_B200_IP ? -acc : __dsub_rn(1.0, acc);
}

__device__ __forceinline__ float4 load_row4(const SearchParams &P, int64_t e, int c, bool u8) {
    if (!u8) return __ldg(reinterpret_cast<const float4 *>(P.vectors + e * P.dim + c));
    uchar4 b = __ldg(reinterpret_cast<const uchar4 *>(P.codes + e * P.dim + c));
    return make_float4(b.x, b.y, b.z, b.w);
}

__device__ __forceinline__ float row_elem(const SearchParams &P, int64_t e, int c, bool u8) {
    return u8 ? float(__ldg(P.codes + e * P.dim + c)) : __ldg(P.vectors + e * P.dim + c);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Float32 warp-cooperative distances for integer-valued data whose partial sums stay below 2^24:
// every product and sum is then exact, in any order, and equals the reference's float64 value.
// Lane j (bit j of umask) receives the distance of the neighbour it holds in `e`.
template <bool U8>
__device__ __forceinline__ void dists_exact_f32(const SearchParams &P, int32_t e, uint32_t umask,
                                                const float *qf, int lane, double &dj) {
    const int dim = P.dim;
    const bool l2 = P.metric == HNSW_B200_L2;
    const bool vec = (dim & 3) == 0;
    while (umask) {
        constexpr int NB = HB_NB_EXACT;  // rows in flight per lane
        int jj[NB];
        int64_t ee[NB];
#pragma unroll
        for (int t = 0; t < NB; t++) {
            if (umask) {
                jj[t] = __ffs(umask) - 1;
                umask &= umask - 1;
            } else {
                jj[t] = -1;
            }
            ee[t] = __shfl_sync(FULL, e, jj[t] < 0 ? 0 : jj[t]);
        }
        float acc[NB];
#pragma unroll
        for (int t = 0; t < NB; t++) acc[t] = 0.f;
        if (vec) {
            for (int c = lane * 4; c < dim; c += 128) {
                float4 qv = *reinterpret_cast<const float4 *>(qf + c);
                float4 xv[NB];
#pragma unroll
                for (int t = 0; t < NB; t++)
                    if (jj[t] >= 0) xv[t] = load_row4(P, ee[t], c, U8);
#pragma unroll
                for (int t = 0; t < NB; t++) {
                    if (jj[t] < 0) continue;
                    if (l2) {
                        float a = xv[t].x - qv.x, b = xv[t].y - qv.y, cc = xv[t].z - qv.z,
                              d = xv[t].w - qv.w;
                        acc[t] = fmaf(a, a, acc[t]);
                        acc[t] = fmaf(b, b, acc[t]);
                        acc[t] = fmaf(cc, cc, acc[t]);
                        acc[t] = fmaf(d, d, acc[t]);
                    } else {
                        acc[t] = fmaf(xv[t].x, qv.x, acc[t]);
                        acc[t] = fmaf(xv[t].y, qv.y, acc[t]);
                        acc[t] = fmaf(xv[t].z, qv.z, acc[t]);
                        acc[t] = fmaf(xv[t].w, qv.w, acc[t]);
                    }
                }
            }
        } else {
            for (int c = lane; c < dim; c += 32) {
                float qv = qf[c];
#pragma unroll
                for (int t = 0; t < NB; t++) {
                    if (jj[t] < 0) continue;
                    float x = row_elem(P, ee[t], c, U8);
                    if (l2) {
                        float a = x - qv;
                        acc[t] = fmaf(a, a, acc[t]);
                    } else {
                        acc[t] = fmaf(x, qv, acc[t]);
                    }
                }
            }
        }
#pragma unroll
        for (int t = 0; t < NB; t++) {
            if (jj[t] < 0) continue;  // uniform
            float s = warp_sum(acc[t]);
            double d = l2 ? double(s) : (P.metric == HNSW_B200_IP ? -double(s) : 1.0 - double(s));
            if (lane == jj[t]) dj = d;
        }
    }
}

// Byte mode: exact integer distances of uint8 rows to a uint8 query, four dimensions per __dp4a
// (|x - q| by __vabsdiffu4 for L2) and one warp reduction instruction per row. Lane j (bit j of
// umask) receives the distance of the neighbour it holds in `e`.
__device__ __forceinline__ void dists_bytes(const SearchParams &P, int32_t e, uint32_t umask,
                                            const uint32_t *q4, int lane, double &dj) {
    const int words = P.dim >> 2;
    const bool l2 = P.metric == HNSW_B200_L2;
    const uint32_t *rows = reinterpret_cast<const uint32_t *>(P.rows8);
    constexpr int NB = HB_NB_BYTES;  // rows in flight per lane
    if (words <= 32) {
        // One word of every row per lane: loads of up to NB rows in flight, then one reduction each.
        const uint32_t q = lane < words ? q4[lane] : 0u;
        while (umask) {
            uint32_t x[NB];
            uint32_t m = umask;
#pragma unroll
            for (int t = 0; t < NB; t++) {
                if (m) {
                    const int j = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t ej = uint32_t(__shfl_sync(FULL, e, j));
                    x[t] = lane < words ? __ldg(rows + size_t(ej) * words + lane) : 0u;
                }
            }
#pragma unroll
            for (int t = 0; t < NB; t++) {
                if (umask) {  // uniform
                    const int j = __ffs(umask) - 1;
                    umask &= umask - 1;
                    uint32_t a;
                    if (l2) {
                        const uint32_t d = __vabsdiffu4(x[t], q);
                        a = __dp4a(d, d, 0u);
                    } else {
                        a = __dp4a(x[t], q, 0u);
                    }
                    const uint32_t sum = __reduce_add_sync(FULL, a);
                    if (lane == j) dj = l2 ? double(sum) : -double(sum);
                }
            }
        }
        return;
    }
    while (umask) {  // wide rows: NB / 2 rows at a time, every lane striding over the words
        constexpr int NW = NB / 2;
        int jj[NW];
        uint32_t acc[NW];
#pragma unroll
        for (int t = 0; t < NW; t++) {
            jj[t] = -1;
            acc[t] = 0u;
            if (umask) {
                jj[t] = __ffs(umask) - 1;
                umask &= umask - 1;
            }
        }
        for (int w = lane; w < words; w += 32) {
            const uint32_t q = q4[w];
#pragma unroll
            for (int t = 0; t < NW; t++) {
                if (jj[t] < 0) continue;
                const uint32_t ej = uint32_t(__shfl_sync(FULL, e, jj[t]));
                const uint32_t x = __ldg(rows + size_t(ej) * words + w);
                if (l2) {
                    const uint32_t d = __vabsdiffu4(x, q);
                    acc[t] = __dp4a(d, d, acc[t]);
                } else {
                    acc[t] = __dp4a(x, q, acc[t]);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < NW; t++) {
            if (jj[t] < 0) continue;  // uniform
            const uint32_t sum = __reduce_add_sync(FULL, acc[t]);
            if (lane == jj[t]) dj = l2 ? double(sum) : -double(sum);
        }
    }
}

// Distance of one node held uniformly by the warp.
template <int MODE, bool U8, class Cx>
__device__ __forceinline__ double dist_one(const SearchParams &P, Cx &C, int32_t e) {
    double d = 0.0;
    if (MODE == MODE_BYTES) {
        dists_bytes(P, e, 1u, C.q4, C.lane, d);
    } else if (MODE == MODE_EXACT) {
        dists_exact_f32<U8>(P, e, 1u, C.qf, C.lane, d);
    } else if (C.lane == 0) {
        d = dist_seq_f64<U8>(P, e, C.qd);
    }
    return __shfl_sync(FULL, d, 0);
}

// Mark one chunk of up to 32 neighbours visited (first occurrence in stored order wins). Returns
// the mask of lanes holding a newly visited neighbour.
// log2 > 0: the open-addressing hash of the upper layers; log2 == 0: the layer-0 bitmap (one
// atomicOr per neighbour, no probing), whose marked ids are listed so they can be cleared.
template <class Cx>
__device__ __forceinline__ uint32_t mark_chunk(const SearchParams &P, Cx &C, int32_t e, int log2,
                                               int &vis_count) {
    const bool has = e >= 0;
    const uint32_t hmask = __ballot_sync(FULL, has);
    int ins = 0;
    if (has) {
        uint32_t same = __match_any_sync(hmask, e);
        if (__ffs(same) - 1 == C.lane) {
            if (log2 > 0) {
                ins = vis_insert(C.vis, log2, e);
            } else {
                const uint32_t bit = 1u << (e & 31);
                ins = (atomicOr(C.vbits + (e >> 5), bit) & bit) ? 0 : 1;
            }
        }
    }
    const uint32_t umask = __ballot_sync(FULL, ins == 1);
    if (log2 > 0) {
        if (__any_sync(FULL, ins < 0)) C.status |= ST_VISITED;
    } else if (umask) {
        const int o = C.vlist_n + __popc(umask & ((1u << C.lane) - 1u));
        if (ins == 1 && o < P.vlist_cap) C.vlist[o] = e;
        C.vlist_n += __popc(umask);
    }
    vis_count += __popc(umask);
    return umask;
}

// Layer-0 bitmap: mark the entry node.
template <class Cx>
__device__ __forceinline__ void bitmap_begin(const SearchParams &P, Cx &C, int32_t e0) {
    C.vlist_n = 1;
    if (C.lane == 0) {
        atomicOr(C.vbits + (e0 >> 5), 1u << (e0 & 31));
        if (P.vlist_cap > 0) C.vlist[0] = e0;
    }
    __syncwarp();
}

// Layer-0 bitmap: return every bit this query set to zero (listed words, or the whole bitmap when
// the list overflowed), so the next query starts from an empty set.
template <class Cx>
__device__ __forceinline__ void bitmap_clear(const SearchParams &P, Cx &C) {
    __syncwarp();
    if (C.vlist_n <= P.vlist_cap) {
        for (int i = C.lane; i < C.vlist_n; i += 32) C.vbits[C.vlist[i] >> 5] = 0u;
    } else {
        int4 *w4 = reinterpret_cast<int4 *>(C.vbits);
        const int64_t n4 = P.vbits_stride >> 2;
        for (int64_t i = C.lane; i < n4; i += 32) w4[i] = make_int4(0, 0, 0, 0);
    }
    __syncwarp();
}

// Distances of the newly visited neighbours: lane j (bit j of umask) receives its distance in dj.
template <int MODE, bool U8, class Cx>
__device__ __forceinline__ void score_chunk(const SearchParams &P, Cx &C, int32_t e, uint32_t umask,
                                            typename Cx::dist_t &dj) {
    double d = 0.0;
    if (MODE == MODE_BYTES) {
        dists_bytes(P, e, umask, C.q4, C.lane, d);
    } else if (MODE == MODE_EXACT) {
        dists_exact_f32<U8>(P, e, umask, C.qf, C.lane, d);
    } else if ((umask >> C.lane) & 1u) {
        d = dist_seq_f64<U8>(P, e, C.qd);
    }
    dj = typename Cx::dist_t(d);
}

// Distance of a byte row held in registers (v4 16-byte words) to the byte query in shared memory:
// L2 sums |x - q|^2 by __vabsdiffu4 + __dp4a, inner product sums x.q by __dp4a. Four independent
// integer accumulators (one per 32-bit word of a 16-byte load) keep the dependent chain at a
// quarter of its length; integer sums, so the value is the same in any order.
template <typename D, class Cx>
__device__ __forceinline__ D row_dot_bytes(const SearchParams &P, const Cx &C, const uint4 (&x)[8],
                                           int v4) {
    const uint4 *qv = reinterpret_cast<const uint4 *>(C.q4);
    uint32_t a0 = 0u, a1 = 0u, a2 = 0u, a3 = 0u;
    if (P.metric == HNSW_B200_L2) {
#pragma unroll
        for (int t = 0; t < 8; t++) {
            if (t < v4) {
                const uint4 q = qv[t];
                const uint32_t d0 = __vabsdiffu4(x[t].x, q.x), d1 = __vabsdiffu4(x[t].y, q.y);
                const uint32_t d2 = __vabsdiffu4(x[t].z, q.z), d3 = __vabsdiffu4(x[t].w, q.w);
                a0 = __dp4a(d0, d0, a0);
                a1 = __dp4a(d1, d1, a1);
                a2 = __dp4a(d2, d2, a2);
                a3 = __dp4a(d3, d3, a3);
            }
        }
        return D((a0 + a1) + (a2 + a3));
    }
#pragma unroll
    for (int t = 0; t < 8; t++) {
        if (t < v4) {
            const uint4 q = qv[t];
            a0 = __dp4a(x[t].x, q.x, a0);
            a1 = __dp4a(x[t].y, q.y, a1);
            a2 = __dp4a(x[t].z, q.z, a2);
            a3 = __dp4a(x[t].w, q.w, a3);
        }
    }
    return -D((a0 + a1) + (a2 + a3));
}

// Byte rows of at most 128 bytes starting on 16-byte boundaries (dim a multiple of 16): every lane
// loads the whole row of the neighbour it holds -- eight 16-byte loads in flight per lane -- before
// the visited marks are resolved, so the gather overlaps the marking atomics and all rows of a chunk
// arrive in one memory round trip. Rows of neighbours found already visited are dropped unscored and
// uncounted. Each lane then sums its own row against the query (shared-memory broadcast reads):
// integer arithmetic, so the value equals dists_bytes' bit for bit.
template <class Cx>
__device__ __forceinline__ uint32_t mark_score_lane_rows(const SearchParams &P, Cx &C, int32_t e,
                                                         int log2, int &vis_count,
                                                         typename Cx::dist_t &dj) {
    using D = typename Cx::dist_t;
    const int v4 = P.dim >> 4;
    const uint4 *row = reinterpret_cast<const uint4 *>(P.rows8 + int64_t(e < 0 ? 0 : e) * P.dim);
    uint4 x[8];
#pragma unroll
    for (int t = 0; t < 8; t++) x[t] = (e >= 0 && t < v4) ? __ldg(row + t) : make_uint4(0u, 0u, 0u, 0u);
    const uint32_t um = mark_chunk(P, C, e, log2, vis_count);
    dj = D(0);
    if ((um >> C.lane) & 1u) dj = row_dot_bytes<D>(P, C, x, v4);
    return um;
}

// Byte rows of exactly 128 bytes, gathered a row per group of eight lanes: in load t, lane l
// fetches 16-byte piece l & 7 of the row held by lane 4t + (l >> 3), so each load instruction
// touches four 128-byte lines instead of 32 and the L1 serves a chunk's rows in an eighth of the
// wavefronts. The loads are issued before the visited marks resolve, as in mark_score_lane_rows.
// Each lane sums its eight pieces against the matching piece of the query; three exchange rounds
// over the group leave lane (g, p) with the whole sum of row 4p + g, and one shuffle hands it to
// the lane holding that neighbour. Integer sums, so the values equal row_dot_bytes' bit for bit.
// (A form for any row of at most 128 bytes, with the pieces beyond the row predicated off and the
// row offset multiplied by dim, measured slower than the row-per-lane gather on the 1M mixture:
// 3.35 against 3.28 ms at ef = 192; this one takes 2.95 ms.)
template <class Cx>
__device__ __forceinline__ uint32_t mark_score_group_rows(const SearchParams &P, Cx &C, int32_t e,
                                                          int log2, int &vis_count,
                                                          typename Cx::dist_t &dj) {
    using D = typename Cx::dist_t;
    const int lane = C.lane;
    const int g = lane >> 3, p = lane & 7;
    uint4 x[8];
#pragma unroll
    for (int t = 0; t < 8; t++) {
        // a lane with no neighbour lends row 0: its sum lands in a slot nobody reads
        const uint32_t et = uint32_t(max(__shfl_sync(FULL, e, 4 * t + g), 0));
        x[t] = __ldg(reinterpret_cast<const uint4 *>(P.rows8 + (uint64_t(et) << 7)) + p);
    }
    const uint32_t um = mark_chunk(P, C, e, log2, vis_count);
    const uint4 q = reinterpret_cast<const uint4 *>(C.q4)[p];
    uint32_t s[8];
    if (P.metric == HNSW_B200_L2) {
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const uint32_t d0 = __vabsdiffu4(x[t].x, q.x), d1 = __vabsdiffu4(x[t].y, q.y);
            const uint32_t d2 = __vabsdiffu4(x[t].z, q.z), d3 = __vabsdiffu4(x[t].w, q.w);
            s[t] = __dp4a(d0, d0, 0u) + __dp4a(d1, d1, 0u) + __dp4a(d2, d2, 0u) + __dp4a(d3, d3, 0u);
        }
    } else {
#pragma unroll
        for (int t = 0; t < 8; t++)
            s[t] = __dp4a(x[t].x, q.x, 0u) + __dp4a(x[t].y, q.y, 0u) + __dp4a(x[t].z, q.z, 0u) +
                   __dp4a(x[t].w, q.w, 0u);
    }
    // Reduce-scatter over the group (lanes that differ in bits 0-2): round b keeps the half of the
    // rows selected by lane bit b and adds the partner's partial sums of that half.
    const bool b2 = lane & 4, b1 = lane & 2, b0 = lane & 1;
    uint32_t h[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
        h[j] = (b2 ? s[4 + j] : s[j]) + __shfl_xor_sync(FULL, b2 ? s[j] : s[4 + j], 4);
    uint32_t w[2];
#pragma unroll
    for (int j = 0; j < 2; j++)
        w[j] = (b1 ? h[2 + j] : h[j]) + __shfl_xor_sync(FULL, b1 ? h[j] : h[2 + j], 2);
    const uint32_t tot = (b0 ? w[1] : w[0]) + __shfl_xor_sync(FULL, b0 ? w[0] : w[1], 1);
    const uint32_t mine = __shfl_sync(FULL, tot, ((lane & 3) << 3) | (lane >> 2));
    dj = D(0);
    if ((um >> lane) & 1u) dj = P.metric == HNSW_B200_L2 ? D(mine) : -D(mine);
    return um;
}

__device__ __forceinline__ void cp_async16(const void *smem_dst, const void *gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
                 "l"(gmem_src)
                 : "memory");
}

// mark_score_lane_rows with the rows staged in shared memory: each lane copies its neighbour's row
// into its own staging slot with 16-byte cp.async (16-byte chunk t of lane l lands at chunk
// t ^ (l & 7) of the slot, so the later reads of a quarter-warp hit distinct banks), resolves the
// visited marks while the copies fly, waits for its own copies, then sums from shared memory.
// Each lane reads only what it copied, so no warp barrier is needed. Same integers as the register
// version.
template <class Cx>
__device__ __forceinline__ uint32_t mark_score_lane_rows_staged(const SearchParams &P, Cx &C,
                                                                int32_t e, int log2, int &vis_count,
                                                                typename Cx::dist_t &dj) {
    using D = typename Cx::dist_t;
    const int v4 = P.dim >> 4;
    const int sw = v4 == 8 ? (C.lane & 7) : 0;
    unsigned char *mine = C.stage + C.lane * P.dim;
    if (e >= 0) {
        const unsigned char *row = P.rows8 + int64_t(e) * P.dim;
#pragma unroll
        for (int t = 0; t < 8; t++)
            if (t < v4) cp_async16(mine + ((t ^ sw) << 4), row + (t << 4));
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    const uint32_t um = mark_chunk(P, C, e, log2, vis_count);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    dj = D(0);
    if ((um >> C.lane) & 1u) {
        const uint4 *xs = reinterpret_cast<const uint4 *>(mine);
        uint4 x[8];
#pragma unroll
        for (int t = 0; t < 8; t++) x[t] = t < v4 ? xs[t ^ sw] : make_uint4(0u, 0u, 0u, 0u);
        dj = row_dot_bytes<D>(P, C, x, v4);
    }
    return um;
}

// Mark a chunk visited and score its new neighbours (lane j of the returned mask gets dj).
template <int MODE, bool U8, int CFG, class Cx>
__device__ __forceinline__ uint32_t mark_and_score(const SearchParams &P, Cx &C, int32_t e, int log2,
                                                   int &vis_count, typename Cx::dist_t &dj) {
    if (MODE == MODE_BYTES && HB_LANE_ROWS && C.lane_rows) {
        // stage_bytes() gives every lane-row search of a byte kernel its staging slot
        if constexpr (cfg_stage(CFG)) return mark_score_lane_rows_staged(P, C, e, log2, vis_count, dj);
        if (HB_GROUP_ROWS && P.dim == 128) return mark_score_group_rows(P, C, e, log2, vis_count, dj);
        return mark_score_lane_rows(P, C, e, log2, vis_count, dj);
    }
    const uint32_t um = mark_chunk(P, C, e, log2, vis_count);
    score_chunk<MODE, U8>(P, C, e, um, dj);
    return um;
}

__device__ __forceinline__ const int32_t *node_links(const SearchParams &P, int32_t c, int layer,
                                                     int &cnt, int &stride) {
    if (layer == 0) {
        cnt = __ldg(P.count0 + c);
        stride = P.links0_stride;
        return P.links0 + int64_t(c) * P.links0_stride;
    }
    int64_t row = __ldg(P.upper_offset + c) + layer - 1;
    cnt = __ldg(P.count_up + row);
    stride = P.links_up_stride;
    return P.links_up + row * P.links_up_stride;
}

// The first chunk of a link row: every lane below the row stride loads its slot in the same round
// trip as the count (slots past the count are ignored), so the count does not gate the load.
__device__ __forceinline__ int32_t first_link(const int32_t *nb, int stride, int cnt, int lane) {
    const int32_t v = lane < stride ? __ldg(nb + lane) : -1;
    return lane < cnt ? v : -1;
}

// ------------------------------------------------------------------------ learned early termination
// Warp matvec of the 12 -> 64 -> 64 -> 1 ReLU network: BF16 weights, FP32 accumulation. Every lane
// holds the same (uniform) features; lane j computes hidden units j and j + 32.
template <class Cx>
__device__ __forceinline__ float mlp_eval(const Cx &C, const float (&raw)[STOP_FEATURES]) {
    const int lane = C.lane;
    const __nv_bfloat162 *w1 = reinterpret_cast<const __nv_bfloat162 *>(C.mlp_w);  // [i][l]
    const __nv_bfloat162 *w2 = w1 + STOP_FEATURES * 32;                              // [i][l]
    const __nv_bfloat162 *w3 = w2 + STOP_HIDDEN * 32;                                // [l]
    const float *b1 = C.mlp_b, *b2 = b1 + STOP_HIDDEN, *b3 = b2 + STOP_HIDDEN;
    const float *mu = b3 + 1, *inv_sd = mu + STOP_FEATURES;
    float f[STOP_FEATURES];
#pragma unroll
    for (int i = 0; i < STOP_FEATURES; i++) f[i] = (raw[i] - mu[i]) * inv_sd[i];
    // lane l computes hidden units l (a) and l + 32 (b)
    float ha = b1[lane], hb = b1[lane + 32];
#pragma unroll
    for (int i = 0; i < STOP_FEATURES; i++) {
        const float2 w = __bfloat1622float2(w1[i * 32 + lane]);
        ha = fmaf(w.x, f[i], ha);
        hb = fmaf(w.y, f[i], hb);
    }
    ha = fmaxf(ha, 0.f);
    hb = fmaxf(hb, 0.f);
    float ga = b2[lane], gb = b2[lane + 32];
#pragma unroll 8
    for (int i = 0; i < 32; i++) {
        const float x = __shfl_sync(FULL, ha, i);  // hidden unit i
        const float y = __shfl_sync(FULL, hb, i);  // hidden unit i + 32
        const float2 wx = __bfloat1622float2(w2[i * 32 + lane]);
        const float2 wy = __bfloat1622float2(w2[(i + 32) * 32 + lane]);
        ga = fmaf(wx.x, x, ga);
        gb = fmaf(wx.y, x, gb);
        ga = fmaf(wy.x, y, ga);
        gb = fmaf(wy.y, y, gb);
    }
    ga = fmaxf(ga, 0.f);
    gb = fmaxf(gb, 0.f);
    const float2 w = __bfloat1622float2(w3[lane]);
    float o = w.x * ga + w.y * gb;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) o += __shfl_xor_sync(FULL, o, off);
    return o + b3[0];
}

// Search-progress state of layer 0 for the stop features.
struct StopState {
    int hops0;        // layer-0 expansions
    int churn;        // admissions into the first k results since the last checkpoint
    int cp;           // checkpoints taken
    int stale;        // consecutive checkpoints without a change of the first k results
    float dk_prev, dk_prev2, d_entry;
};

// At a checkpoint: features, optional trace row, optional network decision (true = stop).
template <class Cx>
__device__ __forceinline__ bool stop_checkpoint(const SearchParams &P, Cx &C, StopState &S, int r,
                                                int scan, typename Cx::dist_t W) {
    const int lane = C.lane;
    const int kk = min(r, P.k);
    const float dk = log1pf(float(C.Rd[kk - 1]));
    const float d1 = log1pf(float(C.Rd[0]));
    // Frontier: distance of the next candidate the search would expand (the worst if none).
    double dn = double(W);
    for (int b = scan; b < r; b += 32) {
        const int i = b + lane;
        const uint32_t m = __ballot_sync(FULL, i < r && !(C.Ri[i] & EXP_BIT));
        if (m) {
            dn = double(C.Rd[b + __ffs(m) - 1]);
            break;
        }
    }
    // Unexpanded entries among the first k results (pending candidates that could still improve
    // the top k), and stagnation of the first k.
    const int unexp = __popc(__ballot_sync(FULL, lane < kk && !(C.Ri[min(lane, kk - 1)] & EXP_BIT)));
    S.stale = S.churn == 0 ? S.stale + 1 : 0;
    float f[STOP_FEATURES];
    f[0] = d1;
    f[1] = dk;
    f[2] = (S.cp > 0 ? S.dk_prev : S.d_entry) - dk;
    f[3] = (S.cp > 1 ? S.dk_prev2 : S.d_entry) - dk;
    f[4] = float(S.hops0) * (1.f / 64.f);
    f[5] = float(C.ndist) * (1.f / 1024.f);
    f[6] = S.d_entry;
    f[7] = float(unexp) / float(max(P.k, 1));
    f[8] = dk - S.d_entry;
    f[9] = float(S.stale) * 0.25f;
    f[10] = float(S.churn) * (1.f / STOP_EVERY);
    f[11] = log1pf(float(dn)) - dk;
    if (P.trace_feat && S.cp < P.trace_cap) {
        if (lane == 0) {
            float *row = P.trace_feat + (int64_t(C.q) * P.trace_cap + S.cp) * STOP_FEATURES;
#pragma unroll
            for (int i = 0; i < STOP_FEATURES; i++) row[i] = f[i];
        }
        if (lane < P.trace_k)
            P.trace_dk[(int64_t(C.q) * P.trace_cap + S.cp) * P.trace_k + lane] =
                lane < r ? double(C.Rd[lane]) : double(INFINITY);
    }
    S.cp++;
    S.dk_prev2 = S.dk_prev;
    S.dk_prev = dk;
    S.churn = 0;
    if (C.mlp_w && r >= P.k) {
        // The threshold rises with the expansions spent: the batch ends with its longest queries,
        // whose late expansions add the least recall for their time.
        const float thr = P.stop_threshold +
                          P.stop_slope * float(max(0, S.hops0 - P.stop_slope_from)) * (1.f / 64.f);
        return mlp_eval(C, f) < thr;
    }
    return false;
}

// ------------------------------------------------------------------------- unfiltered layer search
// Algorithm 2 with exact reference semantics. On entry R[0] holds the single entry node
// (unexpanded) and r == 1; on exit R[0..r) is the sorted result list.
// Admission of one chunk of new neighbours into the sorted results R (unfiltered layer), with the
// same final R, tie stack and expansion frontier as admitting them one by one in stored order.
//
// Sequentially, neighbour j is admitted iff |R| < ef or d_j < W, W the running worst. W is the
// ef-th smallest distance of R0 (R before the chunk) together with every earlier neighbour of the
// chunk, admitted or not: a rejected or evicted one is never below the worst that followed. Hence
//   admitted_j  <=>  #{x in R0 : x.d <= d_j} + #{i < j in the chunk : d_i <= d_j} < ef,
// which every lane evaluates for its own neighbour at once. Inserting with eviction of the maximum
// keeps the ef smallest (distance, id) pairs, so the new R is the first ef entries of R0 merged
// with the admitted set. The evicted entries are the merged tail; the tie stack keeps its entries
// only if the worst distance did not drop, and gains the unexpanded evicted entries that tie the
// final worst, pushed in descending (distance, id) order as the evictions would have pushed them.
// churn (a stop feature) counts admissions that entered the first k at their insertion time.
template <class Cx>
__device__ __forceinline__ void admit_chunk(const SearchParams &P, Cx &C, int32_t e,
                                            typename Cx::dist_t dj, uint32_t um, int ef, int &r,
                                            typename Cx::dist_t &W, int &scan, int &tn, int &churn) {
    using D = typename Cx::dist_t;
    const int lane = C.lane;
    const int r0 = r;
    const D W0 = W;
    const uint32_t cm = __ballot_sync(FULL, ((um >> lane) & 1u) && (r0 < ef || dj < W0));
    if (!cm) return;
    const bool inc = (cm >> lane) & 1u;
    int lo = 0, n_eq = 0, eq_lt = 0;
    if (inc) {
#if HB_UNIFORM_RANK
        // lo: entries of R0 with distance below dj (the same step count in every lane)
        const int a = uniform_prefix(r0, [&](int i) { return C.Rd[i] < dj; });
#else
        int a = 0, b = r0;  // lo: entries of R0 with distance below dj
        while (a < b) {
            const int m = (a + b) >> 1;
            if (C.Rd[m] < dj) a = m + 1;
            else b = m;
        }
#endif
        lo = a;
        if (a < r0 && C.Rd[a] == dj) {  // equal distances (rare): rank by original id
            const int32_t eo = orig_id(P, e);
            for (int i = a; i < r0 && C.Rd[i] == dj; i++) {
                n_eq++;
                eq_lt += orig_id(P, C.Ri[i] & ID_MASK) < eo;
            }
        }
    }
#if HB_ADMIT_MASKS
    // One pass over the candidates: the ones below mine by (distance, id), and the earlier ones at
    // or below my distance, as lane masks.
    uint32_t ltm = 0u, plem = 0u, teq = 0u;  // teq: other candidates at my distance
    for (uint32_t m = cm; m;) {
        const int i = __ffs(m) - 1;
        m &= m - 1;
        const D di = __shfl_sync(FULL, dj, i);
        const uint32_t bit = 1u << i;
        ltm |= di < dj ? bit : 0u;
        teq |= (di == dj && i != lane) ? bit : 0u;
        plem |= (i < lane && di <= dj) ? bit : 0u;
    }
    if (__any_sync(FULL, teq != 0u)) {  // rare: equal distances order by original id
        const int32_t eo = inc ? orig_id(P, e) : -1;
        for (uint32_t m = cm; m;) {
            const int i = __ffs(m) - 1;
            m &= m - 1;
            const int32_t oi = __shfl_sync(FULL, eo, i);
            ltm |= ((teq >> i) & 1u) && oi < eo ? 1u << i : 0u;
        }
    }
    const bool adm = inc && lo + n_eq + __popc(plem) < ef;
    const uint32_t A = __ballot_sync(FULL, adm);
    if (!A) return;
    // admitted pairs below mine: all of them, and earlier ones
    const int rank_a = __popc(ltm & A);
    const int rank_prev = __popc(ltm & A & ((1u << lane) - 1u));
#else
    int prev_le = 0;  // earlier candidates of the chunk at or below dj
    for (uint32_t m = cm; m;) {
        const int i = __ffs(m) - 1;
        m &= m - 1;
        const D di = __shfl_sync(FULL, dj, i);
        prev_le += (i < lane && di <= dj);
    }
    const bool adm = inc && lo + n_eq + prev_le < ef;
    const uint32_t A = __ballot_sync(FULL, adm);
    if (!A) return;
    int rank_a = 0, rank_prev = 0;  // admitted pairs below mine: all of them, and earlier ones
    for (uint32_t m = A; m;) {
        const int i = __ffs(m) - 1;
        m &= m - 1;
        const D di = __shfl_sync(FULL, dj, i);
        const int32_t ii = __shfl_sync(FULL, e, i);
        const bool lt = di < dj || (di == dj && i != lane && pair_lt_int(P, di, ii, dj, e));
        rank_a += lt;
        rank_prev += (lt && i < lane);
    }
#endif
    const int pos_r0 = lo + eq_lt;  // entries of R0 below (dj, e)
    const int fpos = pos_r0 + rank_a;
    churn += __popc(__ballot_sync(FULL, adm && pos_r0 + rank_prev < P.k));
    const int pmin = __reduce_min_sync(FULL, adm ? pos_r0 : 0x7fffffff);
    const int fmin = __reduce_min_sync(FULL, adm ? fpos : 0x7fffffff);
    // Move R0[p] (p >= pmin) up by the admitted entries that precede it, two chunks of 32 at a
    // time, highest first: every entry of a step is read before any is written, and the writes
    // land above every index the next step reads.
    for (int top = r0 - 1; top >= pmin; top -= 64) {
        const int p1 = top - lane, p2 = top - 32 - lane;
        const bool a1 = p1 >= pmin, a2 = p2 >= pmin;
        D d1 = D(0), d2 = D(0);
        int32_t i1 = 0, i2 = 0;
        if (a1) {
            d1 = C.Rd[p1];
            i1 = C.Ri[p1];
        }
        if (a2) {
            d2 = C.Rd[p2];
            i2 = C.Ri[p2];
        }
        int s1 = 0, s2 = 0;
        for (uint32_t m = A; m;) {
            const int i = __ffs(m) - 1;
            m &= m - 1;
            const int pr = __shfl_sync(FULL, pos_r0, i);
            s1 += pr <= p1;
            s2 += pr <= p2;
        }
        __syncwarp();
        if (a1) {
            C.Rd[p1 + s1] = d1;
            C.Ri[p1 + s1] = i1;
        }
        if (a2) {
            C.Rd[p2 + s2] = d2;
            C.Ri[p2 + s2] = i2;
        }
        __syncwarp();
    }
    if (adm) {
        C.Rd[fpos] = dj;
        C.Ri[fpos] = e;
    }
    __syncwarp();
    int rn = r0 + __popc(A);
    if (rn > ef) {
        const int nev = rn - ef;  // at most 32
        const D wf = C.Rd[ef - 1];
        if (r0 == ef && wf != W0) tn = 0;  // the worst dropped: earlier ties are too far now
        bool push = false;
        int32_t pid = 0;
        if (lane < nev) {
            pid = C.Ri[ef + lane] & ID_MASK;
            push = C.Rd[ef + lane] == wf && !(C.Ri[ef + lane] & EXP_BIT);
        }
        const uint32_t pm = __ballot_sync(FULL, push);
        const int idx = tn + __popc(pm >> lane) - 1;  // the largest pair was evicted (pushed) first
        if (push && idx < P.tie_cap) C.ties[idx] = pid;
        tn += __popc(pm);
        if (tn > P.tie_cap) {
            C.status |= ST_TIES;
            tn = P.tie_cap;
        }
        rn = ef;
    }
    __syncwarp();
    r = rn;
    W = C.Rd[r - 1];
    scan = min(scan, fmin);
}

template <int MODE, bool U8, int CFG, class Cx>
__device__ void layer_search(const SearchParams &P, Cx &C, int layer, int ef, int log2, int &r) {
    using D = typename Cx::dist_t;
    const int lane = C.lane;
    if (layer > 0 || (cfg_hash(CFG) && log2 > 0)) {
        vis_clear(C.vis, log2, lane);
        if (lane == 0) vis_insert(C.vis, log2, C.Ri[0] & ID_MASK);
        __syncwarp();
    } else {
        log2 = 0;  // bitmap
        bitmap_begin(P, C, C.Ri[0] & ID_MASK);
    }
    int vis_count = 1;
    const int vis_lim = log2 > 0 ? ((1 << log2) >> 2) * 3 : 0x7fffffff;
    D W = C.Rd[r - 1];
    int scan = 0;  // every result before `scan` is expanded
    int tn = 0;    // tie stack depth
    const bool track = layer == 0 && (P.trace_feat != nullptr || C.mlp_w != nullptr);
    StopState S{0, 0, 0, 0, 0.f, 0.f, log1pf(float(C.Rd[0]))};
    HB_PROF_DECL
    for (;;) {
        HB_PROF(0);
        int32_t c = -1;
        while (scan < r) {
            const int i = scan + lane;
            const bool un = i < r && !(C.Ri[i] & EXP_BIT);
            const uint32_t b = __ballot_sync(FULL, un);
            if (b) {
                const int p = scan + __ffs(b) - 1;
                const int32_t co = C.Ri[p];
                c = co & ID_MASK;
                scan = p + 1;
                __syncwarp();
                if (lane == 0) C.Ri[p] = co | EXP_BIT;
                __syncwarp();
                break;
            }
            scan += 32;
        }
        if (c < 0) {
            if (tn == 0) break;
            tn--;
            c = C.ties[tn];  // ties W (internal ids): expanded after every result
        }
        C.nhops++;
        HB_PROF(1);
        int cnt, stride;
        const int32_t *nb = node_links(P, c, layer, cnt, stride);
        const int32_t e0 = first_link(nb, stride, cnt, lane);
        for (int base = 0; base < cnt; base += 32) {
            const int32_t e = base == 0 ? e0 : (base + lane < cnt ? __ldg(nb + base + lane) : -1);
#ifdef HB_PROFILE
            __syncwarp();
            if (__shfl_sync(FULL, e, 0) == -2) C.status |= 64;  // consume the load before timing
#endif
            HB_PROF(2);
            HB_PROF(3);
            D dj;
            const uint32_t um = mark_and_score<MODE, U8, CFG>(P, C, e, log2, vis_count, dj);
#ifdef HB_PROFILE
            if (__shfl_sync(FULL, dj, 0) == -12345.0) C.status |= 64;  // consume before timing
#endif
            HB_PROF(5);
            C.ndist += __popc(um);
            if (layer == 0 && HB_BATCH_ADMIT) {
                admit_chunk(P, C, e, dj, um, ef, r, W, scan, tn, S.churn);
                HB_PROF(4);
                continue;
            }
            uint32_t am = __ballot_sync(FULL, ((um >> lane) & 1u) && (r < ef || dj < W));
            while (am) {
                const int j = __ffs(am) - 1;
                am &= am - 1;
                const D d = __shfl_sync(FULL, dj, j);
                const int32_t id = __shfl_sync(FULL, e, j);
                if (!(r < ef || d < W)) continue;  // uniform
                const int pos = sorted_rank_int(P, C.Rd, C.Ri, r, d, id, lane);
                shift_up(C.Rd, C.Ri, pos, r, lane);
                if (lane == 0) {
                    C.Rd[pos] = d;
                    C.Ri[pos] = id;
                }
                __syncwarp();
                r++;
                if (pos < P.k) S.churn++;
                if (pos < scan) scan = pos;
                if (r > ef) {  // evict the maximum (d, id)
                    r = ef;
                    const D ed = C.Rd[ef];
                    const int32_t ei = C.Ri[ef];
                    if (ed == C.Rd[ef - 1]) {
                        if (!(ei & EXP_BIT)) {  // still a candidate, tied with the worst
                            if (tn < P.tie_cap) {
                                if (lane == 0) C.ties[tn] = ei & ID_MASK;
                                tn++;
                            } else {
                                C.status |= ST_TIES;
                            }
                        }
                    } else {
                        tn = 0;  // the worst dropped: every tied candidate is now too far
                    }
                }
                W = C.Rd[r - 1];
                if (r == ef) am &= __ballot_sync(FULL, dj < W);
            }
            HB_PROF(4);
        }
        if (vis_count > vis_lim) C.status |= ST_VISITED;
        if (C.status) break;
        if (track && (++S.hops0 % STOP_EVERY) == 0 && stop_checkpoint(P, C, S, r, scan, W)) break;
        HB_PROF(6);
        __syncwarp();
    }
    if (track && P.trace_feat && lane == 0) {
        P.trace_count[C.q] = min(S.cp, P.trace_cap);
        P.trace_hops[C.q] = S.hops0;
    }
}

// -------------------------------------------------------------------- filtered candidate storage
template <typename D>
struct CandsT {
    int s;        // entries in S (descending: S[s-1] is the minimum)
    int g;        // entries in the global spill G
    D gd;         // minimum (d, id) of G when g > 0
    int32_t gi;
};

template <class Cx>
__device__ __forceinline__ void spill_push(const SearchParams &P, Cx &C,
                                           CandsT<typename Cx::dist_t> &K, typename Cx::dist_t d,
                                           int32_t id, int32_t ip) {
    if (K.g < P.spill_cap) {
        if (C.lane == 0) {
            C.spd[K.g] = d;
            C.spi[K.g] = id;
            if (C.spp != C.spi) C.spp[K.g] = ip;
        }
        K.g++;
    } else {
        C.status |= ST_SPILL;
    }
}

// id: original id (ordering); ip: internal id (expansion).
template <class Cx>
__device__ __forceinline__ void cand_push(const SearchParams &P, Cx &C,
                                          CandsT<typename Cx::dist_t> &K, typename Cx::dist_t d,
                                          int32_t id, int32_t ip) {
    using D = typename Cx::dist_t;
    int32_t *sp = C.Sp != C.Si ? C.Sp : nullptr;
    if (K.g > 0 && !pair_lt_raw(d, id, K.gd, K.gi)) {  // not below the spill minimum
        spill_push(P, C, K, d, id, ip);
        return;
    }
    const int pos = count_above(C.Sd, C.Si, K.s, d, id, C.lane);
    shift_up(C.Sd, C.Si, pos, K.s, C.lane, sp);
    if (C.lane == 0) {
        C.Sd[pos] = d;
        C.Si[pos] = id;
        if (sp) sp[pos] = ip;
    }
    __syncwarp();
    K.s++;
    if (K.s > P.s_cap) {  // move the maximum to the spill; it becomes the spill minimum
        const D md = C.Sd[0];
        const int32_t mi = C.Si[0];
        const int32_t mp = sp ? sp[0] : mi;
        shift_down(C.Sd, C.Si, 0, K.s, C.lane, sp);
        K.s--;
        spill_push(P, C, K, md, mi, mp);
        K.gd = md;
        K.gi = mi;
    }
}

// Refill the empty S with the smallest spill entries (at most s_cap / 2), dropping entries that
// can no longer be expanded (distance above the worst of full results).
template <class Cx>
__device__ void cand_refill(const SearchParams &P, Cx &C, CandsT<typename Cx::dist_t> &K, bool prune,
                            typename Cx::dist_t Wp) {
    using D = typename Cx::dist_t;
    const int lane = C.lane;
    const int B = max(1, P.s_cap / 2);
    int32_t *sp = C.Sp != C.Si ? C.Sp : nullptr;
    int s = 0;
    for (int base = 0; base < K.g; base += 32) {
        const int i = base + lane;
        D d = D(0);
        int32_t id = 0, ip = 0;
        bool v = i < K.g;
        if (v) {
            d = C.spd[i];
            id = C.spi[i];
            ip = sp ? C.spp[i] : id;
            if (prune && d > Wp) v = false;
        }
        uint32_t cm = __ballot_sync(FULL, v && (s < B || pair_lt_raw(d, id, C.Sd[0], C.Si[0])));
        while (cm) {
            const int j = __ffs(cm) - 1;
            cm &= cm - 1;
            const D xd = __shfl_sync(FULL, d, j);
            const int32_t xi = __shfl_sync(FULL, id, j);
            const int32_t xp = sp ? __shfl_sync(FULL, ip, j) : xi;
            if (!(s < B || pair_lt_raw(xd, xi, C.Sd[0], C.Si[0]))) continue;
            const int pos = count_above(C.Sd, C.Si, s, xd, xi, lane);
            shift_up(C.Sd, C.Si, pos, s, lane, sp);
            if (lane == 0) {
                C.Sd[pos] = xd;
                C.Si[pos] = xi;
                if (sp) sp[pos] = xp;
            }
            __syncwarp();
            s++;
            if (s > B) {
                shift_down(C.Sd, C.Si, 0, s, lane, sp);
                s--;
            }
            if (s == B) cm &= __ballot_sync(FULL, pair_lt_raw(d, id, C.Sd[0], C.Si[0]));
        }
    }
    // Compact the spill: keep entries not selected (above S's maximum) and not pruned.
    const D td = s > 0 ? C.Sd[0] : -D(INFINITY);
    const int32_t ti = s > 0 ? C.Si[0] : -1;
    int w = 0;
    D md = D(INFINITY);
    int32_t mi = 0x7fffffff;
    for (int base = 0; base < K.g; base += 32) {
        const int i = base + lane;
        D d = D(0);
        int32_t id = 0, ip = 0;
        bool keep = false;
        if (i < K.g) {
            d = C.spd[i];
            id = C.spi[i];
            ip = sp ? C.spp[i] : id;
            keep = !(prune && d > Wp) && pair_lt_raw(td, ti, d, id);
        }
        const uint32_t km = __ballot_sync(FULL, keep);
        __syncwarp();
        if (keep) {
            const int o = w + __popc(km & ((1u << lane) - 1u));
            C.spd[o] = d;
            C.spi[o] = id;
            if (sp) C.spp[o] = ip;
            if (pair_lt_raw(d, id, md, mi)) {
                md = d;
                mi = id;
            }
        }
        w += __popc(km);
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const D od = __shfl_xor_sync(FULL, md, o);
        const int32_t oi = __shfl_xor_sync(FULL, mi, o);
        if (pair_lt_raw(od, oi, md, mi)) {
            md = od;
            mi = oi;
        }
    }
    K.s = s;
    K.g = w;
    K.gd = md;
    K.gi = mi;
}

// ----------------------------------------------------------------------- filtered layer-0 search
// Entries of the descending array [0, m) strictly above (d, id), by one lane (binary search).
template <typename T>
__device__ __forceinline__ int lane_count_above(const T *Ad, const int32_t *Ai, int m, T d,
                                                int32_t id) {
#if HB_UNIFORM_RANK
    return uniform_prefix(m, [&](int i) { return pair_lt_raw(d, id, Ad[i], Ai[i]); });
#else
    int a = 0, b = m;
    while (a < b) {
        const int mid = (a + b) >> 1;
        if (pair_lt_raw(d, id, Ad[mid], Ai[mid])) a = mid + 1;
        else b = mid;
    }
    return a;
#endif
}

// Filtered layer 0: one chunk of new neighbours admitted together, with the same results R, the
// same candidate set (S and the spill) and the same flags as the reference's one-by-one loop
// (numba_engine.py:185-195).
//
// One by one, neighbour j is pushed to the candidates iff |R| < ef or d_j < worst, and also enters
// R when allowed; R changes only by allowed neighbours. As for the unfiltered chunk (admit_chunk),
// R before j is the ef smallest of R0 and the earlier allowed neighbours that passed the first
// test at the chunk's start, so
//   pushed_j  <=>  #{x in R0 : x.d <= d_j} + #{allowed i < j passing : d_i <= d_j} < ef,
// every lane at once; the allowed pushed lanes are R's admissions, merged into R as admit_chunk
// merges (ef smallest (distance, original id) pairs kept). The candidates are a set popped in
// (distance, id) order, and S holds its smallest entries below the spill's minimum, so the
// pushes' order does not matter: the pushes at or above the spill minimum go to the spill; the
// others merge into S, whose largest entries beyond s_cap then go to the spill (their smallest
// becomes the spill minimum), as one-by-one inserts would leave them.
template <class Cx>
__device__ __forceinline__ void admit_chunk_filtered(const SearchParams &P, Cx &C,
                                                     CandsT<typename Cx::dist_t> &K, int32_t e,
                                                     typename Cx::dist_t dj, uint32_t um, int ef,
                                                     int &r, typename Cx::dist_t &W) {
    using D = typename Cx::dist_t;
    const int lane = C.lane;
    const uint32_t below_me = (1u << lane) - 1u;
    const int r0 = r;
    const D W0 = W;
    const uint32_t pm = __ballot_sync(FULL, ((um >> lane) & 1u) && (r0 < ef || dj < W0));
    if (!pm) return;
    const bool inp = (pm >> lane) & 1u;
    const bool al = inp && is_allowed(P.allowed, e);
    const uint32_t AM = __ballot_sync(FULL, al);
    const int32_t eo = inp ? orig_id(P, e) : 0x7fffffff;  // orders R and the candidates
    int lo = 0, n_eq = 0, eq_lt = 0;  // R0 entries below dj, equal to dj, below (dj, eo)
    if (inp) {
#if HB_UNIFORM_RANK
        const int a = uniform_prefix(r0, [&](int i) { return C.Rd[i] < dj; });
#else
        int a = 0, b = r0;
        while (a < b) {
            const int m = (a + b) >> 1;
            if (C.Rd[m] < dj) a = m + 1;
            else b = m;
        }
#endif
        lo = a;
        for (int i = a; i < r0 && C.Rd[i] == dj; i++) {
            n_eq++;
            eq_lt += (C.Ri[i] & ID_MASK) < eo;
        }
    }
    uint32_t plem = 0u, ltm = 0u;  // earlier allowed at or below my distance; allowed below me
    for (uint32_t m = AM; m;) {
        const int i = __ffs(m) - 1;
        m &= m - 1;
        const D di = __shfl_sync(FULL, dj, i);
        const int32_t ii = __shfl_sync(FULL, eo, i);
        const uint32_t bit = 1u << i;
        plem |= (i < lane && di <= dj) ? bit : 0u;
        ltm |= (di < dj || (di == dj && ii < eo)) ? bit : 0u;
    }
    const bool pushed = inp && lo + n_eq + __popc(plem) < ef;
    const uint32_t CM = __ballot_sync(FULL, pushed);
    const uint32_t A = CM & AM;  // R's admissions
    const bool adm = (A >> lane) & 1u;
    if (A) {
        const int pos_r0 = lo + eq_lt;  // R0 entries below (dj, eo)
        const int fpos = pos_r0 + __popc(ltm & A);
        const int pmin = __reduce_min_sync(FULL, adm ? pos_r0 : 0x7fffffff);
        int32_t *rp = C.Rp != C.Ri ? C.Rp : nullptr;
        // Move R0[p] (p >= pmin) up by the admissions before it, two chunks of 32 a step, highest
        // first (every read of a step precedes its writes; writes land above the next step's reads).
        for (int top = r0 - 1; top >= pmin; top -= 64) {
            const int p1 = top - lane, p2 = top - 32 - lane;
            const bool a1 = p1 >= pmin, a2 = p2 >= pmin;
            D d1 = D(0), d2 = D(0);
            int32_t i1 = 0, i2 = 0, q1 = 0, q2 = 0;
            if (a1) {
                d1 = C.Rd[p1];
                i1 = C.Ri[p1];
                if (rp) q1 = rp[p1];
            }
            if (a2) {
                d2 = C.Rd[p2];
                i2 = C.Ri[p2];
                if (rp) q2 = rp[p2];
            }
            int s1 = 0, s2 = 0;
            for (uint32_t m = A; m;) {
                const int i = __ffs(m) - 1;
                m &= m - 1;
                const int pr = __shfl_sync(FULL, pos_r0, i);
                s1 += pr <= p1;
                s2 += pr <= p2;
            }
            __syncwarp();
            if (a1) {
                C.Rd[p1 + s1] = d1;
                C.Ri[p1 + s1] = i1;
                if (rp) rp[p1 + s1] = q1;
            }
            if (a2) {
                C.Rd[p2 + s2] = d2;
                C.Ri[p2 + s2] = i2;
                if (rp) rp[p2 + s2] = q2;
            }
            __syncwarp();
        }
        if (adm) {
            C.Rd[fpos] = dj;
            C.Ri[fpos] = eo;
            if (rp) rp[fpos] = e;
        }
        __syncwarp();
        r = min(ef, r0 + __popc(A));
        W = C.Rd[r - 1];
    }
    // ---- candidates: every pushed lane
    if (!CM) return;
    int32_t *sp = C.Sp != C.Si ? C.Sp : nullptr;
    // at or above the spill minimum: appended to the spill in lane order
    const bool low = pushed && (K.g == 0 || pair_lt_raw(dj, eo, K.gd, K.gi));
    const uint32_t LM = __ballot_sync(FULL, low);
    const uint32_t HM = CM & ~LM;
    if (HM) {
        const int idx = K.g + __popc(HM & below_me);
        if (((HM >> lane) & 1u) && idx < P.spill_cap) {
            C.spd[idx] = dj;
            C.spi[idx] = eo;
            if (C.spp != C.spi) C.spp[idx] = e;
        }
        K.g += __popc(HM);
        if (K.g > P.spill_cap) {
            C.status |= ST_SPILL;
            K.g = P.spill_cap;
        }
    }
    if (!LM) return;
    // below it: merged into S (descending by (distance, original id)); the excess largest of the
    // merge go to the spill
    const int s0 = K.s;
    const int nl = __popc(LM);
    int s_above = low ? lane_count_above(C.Sd, C.Si, s0, dj, eo) : 0;  // S0 entries above mine
    int new_above = 0;  // pushed low lanes above mine
    for (uint32_t m = LM; m;) {
        const int i = __ffs(m) - 1;
        m &= m - 1;
        const D di = __shfl_sync(FULL, dj, i);
        const int32_t ii = __shfl_sync(FULL, eo, i);
        new_above += pair_lt_raw(dj, eo, di, ii);
    }
    const int rank_new = s_above + new_above;  // my index in the merged descending array
    const int excess = max(0, s0 + nl - P.s_cap);
    // S0[p] lies at p + a(p) in the merge, a(p) = pushed entries above it (those with s_above <= p);
    // p + a(p) grows with p, so the evicted S0 entries (merged index below excess) are a prefix.
    int x0 = 0;
    uint32_t E1 = 0u;
    if (excess > 0) {
        int a = 0;  // a(lane)
        for (uint32_t m = LM; m;) {
            const int i = __ffs(m) - 1;
            m &= m - 1;
            a += __shfl_sync(FULL, s_above, i) <= lane;
        }
        const bool ev0 = lane < s0 && lane + a < excess;
        const bool ev1 = low && rank_new < excess;  // pushed entries evicted straight to the spill
        const uint32_t E0 = __ballot_sync(FULL, ev0);
        E1 = __ballot_sync(FULL, ev1);
        x0 = __popc(E0);
        // A lane may hold both an evicted S0 entry (S0[lane]) and its own evicted pushed entry.
        D sd0 = D(0);
        int32_t si0 = 0, sp0 = 0;
        if (ev0) {
            sd0 = C.Sd[lane];
            si0 = C.Si[lane];
            sp0 = sp ? sp[lane] : si0;
            const int idx = K.g + lane;
            if (idx < P.spill_cap) {
                C.spd[idx] = sd0;
                C.spi[idx] = si0;
                if (C.spp != C.spi) C.spp[idx] = sp0;
            }
        }
        if (ev1) {
            const int idx = K.g + x0 + __popc(E1 & below_me);
            if (idx < P.spill_cap) {
                C.spd[idx] = dj;
                C.spi[idx] = eo;
                if (C.spp != C.spi) C.spp[idx] = e;
            }
        }
        // the smallest evicted entry (merged index excess - 1) becomes the spill minimum
        const uint32_t L0 = __ballot_sync(FULL, ev0 && lane + a == excess - 1);
        const uint32_t L1 = __ballot_sync(FULL, ev1 && rank_new == excess - 1);
        const int src = __ffs(L0 ? L0 : L1) - 1;
        const D gd0 = __shfl_sync(FULL, sd0, src), gd1 = __shfl_sync(FULL, dj, src);
        const int32_t gi0 = __shfl_sync(FULL, si0, src), gi1 = __shfl_sync(FULL, eo, src);
        K.gd = L0 ? gd0 : gd1;
        K.gi = L0 ? gi0 : gi1;
        K.g += excess;
        if (K.g > P.spill_cap) {
            C.status |= ST_SPILL;
            K.g = P.spill_cap;
        }
        __syncwarp();
        // S0[x0 ..) down by x0, lowest chunk first (each chunk read before written; writes land
        // below the next chunk's reads)
        if (x0 > 0) {
            for (int base = x0; base < s0; base += 32) {
                const int i = base + lane;
                D d = D(0);
                int32_t id = 0, ip = 0;
                if (i < s0) {
                    d = C.Sd[i];
                    id = C.Si[i];
                    if (sp) ip = sp[i];
                }
                __syncwarp();
                if (i < s0) {
                    C.Sd[i - x0] = d;
                    C.Si[i - x0] = id;
                    if (sp) sp[i - x0] = ip;
                }
                __syncwarp();
            }
        }
    }
    // the remaining pushed entries: inserted into S0' = S0[x0 ..) at ins = s_above - x0, the
    // entries at or after an insertion point moving up by the insertions at or before them
    const uint32_t RM = LM & ~E1;
    const int s1 = s0 - x0;
    if (RM) {
        const bool mine = (RM >> lane) & 1u;
        const int ins = s_above - x0;
        const int pmin = __reduce_min_sync(FULL, mine ? ins : 0x7fffffff);
        for (int top = s1 - 1; top >= pmin; top -= 64) {
            const int p1 = top - lane, p2 = top - 32 - lane;
            const bool a1 = p1 >= pmin, a2 = p2 >= pmin;
            D d1 = D(0), d2 = D(0);
            int32_t i1 = 0, i2 = 0, q1 = 0, q2 = 0;
            if (a1) {
                d1 = C.Sd[p1];
                i1 = C.Si[p1];
                if (sp) q1 = sp[p1];
            }
            if (a2) {
                d2 = C.Sd[p2];
                i2 = C.Si[p2];
                if (sp) q2 = sp[p2];
            }
            int u1 = 0, u2 = 0;
            for (uint32_t m = RM; m;) {
                const int i = __ffs(m) - 1;
                m &= m - 1;
                const int pi = __shfl_sync(FULL, ins, i);
                u1 += pi <= p1;
                u2 += pi <= p2;
            }
            __syncwarp();
            if (a1) {
                C.Sd[p1 + u1] = d1;
                C.Si[p1 + u1] = i1;
                if (sp) sp[p1 + u1] = q1;
            }
            if (a2) {
                C.Sd[p2 + u2] = d2;
                C.Si[p2 + u2] = i2;
                if (sp) sp[p2 + u2] = q2;
            }
            __syncwarp();
        }
        if (mine) {
            const int f = rank_new - excess;
            C.Sd[f] = dj;
            C.Si[f] = eo;
            if (sp) sp[f] = e;
        }
        __syncwarp();
    }
    K.s = s1 + __popc(RM);
}

// numba_engine._search_layer0_filtered (:151-198): results hold allowed nodes only, the worst of
// an empty result list is +inf, and the search stops only when the results are full and the
// closest candidate is strictly farther than the worst.
template <int MODE, bool U8, int CFG, class Cx>
__device__ void layer0_filtered(const SearchParams &P, Cx &C, int ef, int log2, double d0,
                                int32_t e0, int32_t o0, int &r) {
    using D = typename Cx::dist_t;
    const int lane = C.lane;
    log2 = 0;  // bitmap
    bitmap_begin(P, C, e0);
    if (lane == 0) {  // candidates hold internal ids; results hold both
        C.Sd[0] = D(d0);
        C.Si[0] = o0;
        C.Sp[0] = e0;
        if (is_allowed(P.allowed, e0)) {
            C.Rd[0] = D(d0);
            C.Ri[0] = o0;
            C.Rp[0] = e0;
        }
    }
    __syncwarp();
    r = is_allowed(P.allowed, e0) ? 1 : 0;
    CandsT<D> K{1, 0, D(INFINITY), 0x7fffffff};
    int vis_count = 1;
    const int vis_lim = 0x7fffffff;
    D W = r > 0 ? C.Rd[r - 1] : D(INFINITY);
    for (;;) {
        if (K.s == 0) {
            if (K.g == 0) break;
            cand_refill(P, C, K, r == ef, W);
            if (K.s == 0) break;
        }
        const D dc = C.Sd[K.s - 1];
        const int32_t c = C.Sp[K.s - 1];
        K.s--;
        if (r == ef && dc > W) break;
        C.nhops++;
        const int cnt = __ldg(P.count0 + c);
        const int32_t *nb = P.links0 + int64_t(c) * P.links0_stride;
        for (int base = 0; base < cnt; base += 32) {
            const int32_t e = base == 0 ? first_link(nb, P.links0_stride, cnt, lane)
                                        : (base + lane < cnt ? __ldg(nb + base + lane) : -1);
            D dj;
            const uint32_t um = mark_and_score<MODE, U8, CFG>(P, C, e, log2, vis_count, dj);
            C.ndist += __popc(um);
            if (HB_BATCH_ADMIT_FILT) {
                admit_chunk_filtered(P, C, K, e, dj, um, ef, r, W);
                continue;
            }
            const int32_t eo = e >= 0 ? orig_id(P, e) : -1;
            uint32_t am = __ballot_sync(FULL, ((um >> lane) & 1u) && (r < ef || dj < W));
            while (am) {
                const int j = __ffs(am) - 1;
                am &= am - 1;
                const D d = __shfl_sync(FULL, dj, j);
                const int32_t id = __shfl_sync(FULL, e, j);
                const int32_t ido = __shfl_sync(FULL, eo, j);
                if (!(r < ef || d < W)) continue;
                cand_push(P, C, K, d, ido, id);
                if (is_allowed(P.allowed, id)) {
                    const int pos = count_below(C.Rd, C.Ri, r, d, ido, lane);
                    shift_up(C.Rd, C.Ri, pos, r, lane, C.Rp != C.Ri ? C.Rp : nullptr);
                    if (lane == 0) {
                        C.Rd[pos] = d;
                        C.Ri[pos] = ido;
                        C.Rp[pos] = id;
                    }
                    __syncwarp();
                    r++;
                    if (r > ef) r = ef;
                    W = C.Rd[r - 1];
                }
                if (r == ef) am &= __ballot_sync(FULL, dj < W);
            }
        }
        if (vis_count > vis_lim) C.status |= ST_VISITED;
        if (C.status) break;
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------ rerank epilogue
// numba_engine._rerank_batch (:506-530): exact float64 distances from the float32 query to the
// first m beam entries, best k by (distance, id).
// internal: R holds internal ids only (unfiltered); otherwise Ri holds the original ids.
// bytes: the query and the vectors are bytes (P.rerank_rows8, query bytes in C.q4): integer sums.
template <class Cx>
__device__ int rerank_epilogue(const SearchParams &P, Cx &C, int m, bool internal, bool bytes) {
    const int lane = C.lane;
    const int k = P.k;
    int a = 0;
    for (int base = 0; base < m; base += 32) {
        const int i = base + lane;
        const bool has = i < m;
        const int32_t ri = has ? (C.Ri[i] & ID_MASK) : -1;
        const int32_t id = has && internal ? orig_id(P, ri) : ri;  // original id
        double d = INFINITY;
        if (bytes) {
            if (has) {
                const uint4 *row = reinterpret_cast<const uint4 *>(
                    P.rerank_rows8 + int64_t(C.Rp[i] & ID_MASK) * P.dim);
                const int v4 = P.dim >> 4;
                uint4 x[8];
#pragma unroll
                for (int t = 0; t < 8; t++) x[t] = t < v4 ? __ldg(row + t) : make_uint4(0u, 0u, 0u, 0u);
                d = row_dot_bytes<double>(P, C, x, v4);
            }
        } else if (has) {
            d = dist_seq_f64<false>(P, C.Rp[i] & ID_MASK, C.qd);
        }
        uint32_t am = __ballot_sync(FULL, has);
        while (am) {
            const int j = __ffs(am) - 1;
            am &= am - 1;
            const double xd = __shfl_sync(FULL, d, j);
            const int32_t xi = __shfl_sync(FULL, id, j);
            if (a == k && !pair_lt_raw(xd, xi, C.Ad[k - 1], C.Ai[k - 1])) continue;
            const int pos = count_below(C.Ad, C.Ai, a, xd, xi, lane);
            shift_up(C.Ad, C.Ai, pos, a, lane);
            if (lane == 0) {
                C.Ad[pos] = xd;
                C.Ai[pos] = xi;
            }
            __syncwarp();
            a = min(a + 1, k);
        }
    }
    return a;
}

// --------------------------------------------------------------------------------------- kernel
template <int MODE, bool U8, bool FILT, int CFG>
__global__ void __launch_bounds__(WPB * 32, min_blocks<MODE, FILT, CFG>())
    search_kernel(const SearchParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const bool rerank = P.rerank_queries != nullptr;
    const bool two_ids = P.node_ids != nullptr;  // filtered results keep both ids
    const int stage = stage_bytes(MODE, CFG, P.lane_rows, P.dim);
    const size_t wb = warp_smem_bytes(P.ef_cap, P.dim, FILT, P.s_cap, rerank ? P.k : 0, two_ids, stage);
    unsigned char *p = smem + size_t(warp) * wb;
    using D = std::conditional_t<MODE == MODE_BYTES, float, double>;
    CtxT<D> C;
    C.lane = lane;
    C.stage = stage ? p : nullptr;
    p += al16(size_t(stage));
    C.Rd = reinterpret_cast<D *>(p);  // 8 bytes a slot are reserved either way
    p += al16(size_t(result_slots(P.ef_cap)) * 8);
    C.Ri = reinterpret_cast<int32_t *>(p);
    p += al16(size_t(result_slots(P.ef_cap)) * 4);
    C.Rp = C.Ri;  // same ids: one array (reads of Rp mask the expanded bit)
    if (two_ids && FILT) {
        C.Rp = reinterpret_cast<int32_t *>(p);
        p += al16(size_t(result_slots(P.ef_cap)) * 4);
    }
    C.qd = reinterpret_cast<double *>(p);
    p += al16(size_t(P.dim) * 8);
    C.qf = reinterpret_cast<float *>(p);
    p += al16(size_t(P.dim) * 4);
    C.q4 = reinterpret_cast<uint32_t *>(p);
    p += al16(size_t(P.dim));
    C.Sd = nullptr;
    C.Si = nullptr;
    C.Sp = nullptr;
    if (FILT) {
        C.Sd = reinterpret_cast<D *>(p);
        p += al16(size_t(P.s_cap + 1) * 8);
        C.Si = reinterpret_cast<int32_t *>(p);
        p += al16(size_t(P.s_cap + 1) * 4);
        C.Sp = C.Si;
        if (two_ids) {
            C.Sp = reinterpret_cast<int32_t *>(p);
            p += al16(size_t(P.s_cap + 1) * 4);
        }
    }
    C.Ad = reinterpret_cast<double *>(p);
    p += rerank ? al16(size_t(P.k + 1) * 8) : 0;
    C.Ai = reinterpret_cast<int32_t *>(p);
    C.mlp_w = nullptr;
    C.mlp_b = nullptr;
    if (!FILT && P.stop_mlp) {  // block-shared copy of the network after the warp regions
        unsigned char *m = smem + size_t(WPB) * wb;
        const unsigned char *src = static_cast<const unsigned char *>(P.stop_mlp);
        for (int i = threadIdx.x; i < int(MLP_BYTES / 4); i += blockDim.x)
            reinterpret_cast<uint32_t *>(m)[i] = reinterpret_cast<const uint32_t *>(src)[i];
        __syncthreads();
        C.mlp_w = reinterpret_cast<const __nv_bfloat16 *>(m);
        C.mlp_b = reinterpret_cast<const float *>(m + size_t(MLP_BF16) * 2);
    }
    const int64_t slot = int64_t(blockIdx.x) * WPB + warp;
    C.vis = P.vis + slot * P.vis_stride;
    C.vbits = P.vbits + slot * P.vbits_stride;
    C.vlist = P.vlist + slot * P.vlist_cap;
    C.vlist_n = 0;
    C.ties = P.ties + slot * P.tie_cap;
    // byte searches keep float candidates: the first half of each slot of the double spill
    C.spd = FILT ? reinterpret_cast<D *>(P.spill_d + slot * P.spill_cap) : nullptr;
    C.spi = FILT ? P.spill_i + slot * P.spill_cap : nullptr;
    C.spp = FILT ? (two_ids ? P.spill_p + slot * P.spill_cap : C.spi) : nullptr;
    C.lane_rows = P.lane_rows && (P.dim & 15) == 0 && P.dim <= 128;

    for (;;) {
        int w = 0;
        if (lane == 0) w = atomicAdd(P.queue, 1);
        w = __shfl_sync(FULL, w, 0);
        if (w >= P.n_work) break;
        const int q = P.qlist ? P.qlist[w] : w;
        const int dim = P.dim;
        uint8_t *qb = reinterpret_cast<uint8_t *>(C.q4);
        if (P.queries_f64) {
            const double *src = static_cast<const double *>(P.queries) + int64_t(q) * dim;
            for (int i = lane; i < dim; i += 32) {
                C.qd[i] = src[i];
                C.qf[i] = float(src[i]);
                if (MODE == MODE_BYTES) qb[i] = uint8_t(src[i]);
            }
        } else {
            const float *src = static_cast<const float *>(P.queries) + int64_t(q) * dim;
            for (int i = lane; i < dim; i += 32) {
                C.qd[i] = double(src[i]);
                C.qf[i] = src[i];
                if (MODE == MODE_BYTES) qb[i] = uint8_t(src[i]);
            }
        }
        __syncwarp();
        C.ndist = 0;
        C.nhops = 0;
        C.status = 0;
        C.q = q;
#ifdef HB_PROFILE
        for (int i = 0; i < 8; i++) C.prof[i] = 0;
#endif
        if (!FILT && (P.stop_mlp || P.trace_feat)) {
            double ss = 0.0;
            for (int i = lane; i < dim; i += 32) ss += C.qd[i] * C.qd[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(FULL, ss, o);
            C.qfeat = log1pf(float(ss));
        }
        // Entry point, then greedy descent (ef = 1) through the upper layers.
        // layer_search keeps internal ids in Ri (ties order by original id through lookups).
        int32_t e0 = int32_t(P.entry_point);  // internal id
        double d0 = dist_one<MODE, U8>(P, C, e0);
        C.ndist++;
        int r = 1;
        for (int layer = P.max_level; layer > 0 && !C.status; layer--) {
            if (lane == 0) {
                C.Rd[0] = D(d0);
                C.Ri[0] = e0;
            }
            __syncwarp();
            r = 1;
            layer_search<MODE, U8, CFG>(P, C, layer, 1, P.vis_up_log2, r);
            d0 = C.Rd[0];
            e0 = C.Ri[0] & ID_MASK;
            __syncwarp();
        }
        const int ef0 = max(__ldg(P.ef + q), P.k_search);
        if (!C.status) {
            if constexpr (FILT) {
                layer0_filtered<MODE, U8, CFG>(P, C, ef0, P.vis_log2, d0, e0, orig_id(P, e0), r);
            } else {
                if (lane == 0) {
                    C.Rd[0] = D(d0);
                    C.Ri[0] = e0;
                }
                __syncwarp();
                r = 1;
                layer_search<MODE, U8, CFG>(P, C, 0, ef0, P.vis_log2, r);
            }
            bitmap_clear(P, C);
        }
        if (C.status) {
            if (lane == 0) {
                P.status[q] = C.status;
                atomicAdd(P.n_failed, 1);
            }
            __syncwarp();
            continue;
        }
        const int k = P.k;
        int64_t *oi = P.out_ids + int64_t(q) * k;
        double *od = P.out_dists + int64_t(q) * k;
        if (rerank) {
            // A query whose values are all bytes, over byte vectors, is re-scored in integers
            // (its bytes replace the searched query's in C.q4): the float64 sums of the reference
            // are exact on such data, so the distances are the same numbers.
            const float *rq = P.rerank_queries + int64_t(q) * dim;
            uint32_t not_byte = P.rerank_rows8 ? 0u : 1u;
            for (int i = lane; i < dim; i += 32) {
                const float v = rq[i];
                C.qd[i] = double(v);
                if (rintf(v) != v || !(v >= 0.f) || !(v <= 255.f)) not_byte = 1u;
                else if (P.rerank_rows8) qb[i] = uint8_t(v);
            }
            not_byte = __reduce_or_sync(FULL, not_byte);
            __syncwarp();
            const int a = rerank_epilogue(P, C, min(r, P.k_search), !FILT, not_byte == 0u);
            for (int i = lane; i < k; i += 32) {
                oi[i] = i < a ? int64_t(C.Ai[i]) : -1;
                od[i] = i < a ? C.Ad[i] : INFINITY;
            }
        } else {
            for (int i = lane; i < k; i += 32) {
                const int32_t ri = i < r ? (C.Ri[i] & ID_MASK) : -1;
                oi[i] = i < r ? int64_t(FILT ? ri : orig_id(P, ri)) : -1;
                od[i] = i < r ? double(C.Rd[i]) : double(INFINITY);
            }
        }
#ifdef HB_PROFILE
        if (lane == 0)
            for (int i = 0; i < 8; i++) atomicAdd(&hb_prof[i], C.prof[i]);
#endif
        if (lane == 0) {
            P.status[q] = 0;
            if (P.out_ctr) {
                P.out_ctr[2 * int64_t(q)] = C.ndist;
                P.out_ctr[2 * int64_t(q) + 1] = C.nhops;
            }
            if (P.cells) {  // the start order's per-cell cost table; cells outside it are skipped
                const int c = P.cells[q];
                if (c >= 0 && c < P.n_cells) {
                    const int64_t tb = P.stop_mlp ? 1 : 0;
                    atomicAdd(P.cell_cost + tb * P.n_cells + c,
                              double(C.nhops) / double(max(1, __ldg(P.ef + q))));
                    atomicAdd(P.cell_cost + (2 + tb) * P.n_cells + c, 1.0);
                }
            }
        }
        __syncwarp();
    }
}

// Row numbers 0 .. n-1 (the values sorted by priority into the first work list).
__global__ void iota_rows(int32_t *out, int32_t n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = i;
}

// Collect the work items whose status is nonzero into qlist_out (order: by query row).
__global__ void collect_failed(const int32_t *status, const int32_t *qlist, int32_t n_work,
                               int32_t *out, int32_t *n_out) {
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n_work; w += gridDim.x * blockDim.x) {
        const int q = qlist ? qlist[w] : w;
        if (status[q] != 0) out[atomicAdd(n_out, 1)] = q;
    }
}

// ======================================================================================== host
thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                     \
    do {                                                                                   \
        cudaError_t _e = (expr);                                                           \
        if (_e != cudaSuccess)                                                             \
            return fail(HNSW_B200_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

struct Buffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    // Grow to at least `want` bytes; a new allocation is zero-filled when `zero` (on `s`).
    int ensure(size_t want, bool zero = false, cudaStream_t s = nullptr) {
        if (want <= bytes) return 0;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        size_t b = std::max(want, size_t(256));
        if (cudaMalloc(&ptr, b) != cudaSuccess) {
            cudaGetLastError();
            return fail(HNSW_B200_ENOMEM, "cudaMalloc of " + std::to_string(b) + " bytes failed");
        }
        bytes = b;
        if (zero && cudaMemsetAsync(ptr, 0, b, s) != cudaSuccess)
            return fail(HNSW_B200_ECUDA, "cudaMemsetAsync of new scratch failed");
        return 0;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct Handle {
    hnsw_b200_graph_t g;
    int device = 0;
    int sms = 148;
    Buffer counters;  // queue, n_failed, n_list
    Buffer status;
    Buffer qlist[2];  // retry work lists (ping-pong)
    Buffer order_rows, order_keys, order_list, sort_temp;  // start order by priority
    Buffer vis, ties, spill_d, spill_i, spill_p, vbits, vlist;
    bool bits_dirty = false;  // a launch failed mid-flight: bitmaps must be re-zeroed
    int32_t *host_pinned = nullptr;  // 4 ints
    long long launches = 0;
    std::mutex mu;
};

template <int MODE, bool U8, bool FILT, int CFG>
int launch_one(const SearchParams &P, size_t smem_block, int blocks, cudaStream_t s) {
    auto kern = search_kernel<MODE, U8, FILT, CFG>;
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem_block)));
    kern<<<blocks, WPB * 32, smem_block, s>>>(P);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

template <int MODE, bool U8, int CFG>
int launch_cfg(const SearchParams &P, bool filt, size_t smem_block, int blocks, cudaStream_t s) {
    return filt ? launch_one<MODE, U8, true, CFG>(P, smem_block, blocks, s)
                : launch_one<MODE, U8, false, CFG>(P, smem_block, blocks, s);
}

// One launch of the kernel for (mode, rows, filter, configuration); cfg < configs_of(mode).
int dispatch(const SearchParams &P, int mode, bool u8, bool filt, int cfg, size_t smem_block,
             int blocks, cudaStream_t s) {
    if (mode == MODE_BYTES) {
        switch (cfg) {
            case 1: return launch_cfg<MODE_BYTES, true, 1>(P, filt, smem_block, blocks, s);
            case 2: return launch_cfg<MODE_BYTES, true, 2>(P, filt, smem_block, blocks, s);
            case 3: return launch_cfg<MODE_BYTES, true, 3>(P, filt, smem_block, blocks, s);
            default: return launch_cfg<MODE_BYTES, true, 0>(P, filt, smem_block, blocks, s);
        }
    }
    if (mode == MODE_EXACT)
        return u8 ? launch_cfg<MODE_EXACT, true, 0>(P, filt, smem_block, blocks, s)
                  : launch_cfg<MODE_EXACT, false, 0>(P, filt, smem_block, blocks, s);
    return u8 ? launch_cfg<MODE_F64, true, 0>(P, filt, smem_block, blocks, s)
              : launch_cfg<MODE_F64, false, 0>(P, filt, smem_block, blocks, s);
}

template <int MODE, bool U8, bool FILT, int CFG>
int occupancy_of(size_t smem_block, int *blocks_per_sm) {
    auto kern = search_kernel<MODE, U8, FILT, CFG>;
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem_block)));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, WPB * 32,
                                                           smem_block));
    return 0;
}

template <int MODE, bool U8, int CFG>
int occupancy_cfg(bool filt, size_t smem_block, int *bps) {
    return filt ? occupancy_of<MODE, U8, true, CFG>(smem_block, bps)
                : occupancy_of<MODE, U8, false, CFG>(smem_block, bps);
}

int occupancy(int mode, bool u8, bool filt, int cfg, size_t smem_block, int *bps) {
    if (mode == MODE_BYTES) {
        switch (cfg) {
            case 1: return occupancy_cfg<2, true, 1>(filt, smem_block, bps);
            case 2: return occupancy_cfg<2, true, 2>(filt, smem_block, bps);
            case 3: return occupancy_cfg<2, true, 3>(filt, smem_block, bps);
            default: return occupancy_cfg<2, true, 0>(filt, smem_block, bps);
        }
    }
    if (mode == MODE_EXACT)
        return u8 ? occupancy_cfg<1, true, 0>(filt, smem_block, bps)
                  : occupancy_cfg<1, false, 0>(filt, smem_block, bps);
    return u8 ? occupancy_cfg<0, true, 0>(filt, smem_block, bps)
              : occupancy_cfg<0, false, 0>(filt, smem_block, bps);
}

int ilog2_ceil(int64_t x) {
    int l = 0;
    while ((int64_t(1) << l) < x) l++;
    return l;
}

}  // namespace hb

using namespace hb;

extern "C" {

#ifdef HB_PROFILE
int hnsw_b200_prof_read(unsigned long long *out, int reset) {
    cudaMemcpyFromSymbol(out, hb::hb_prof, sizeof(unsigned long long) * 8);
    if (reset) {
        unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        cudaMemcpyToSymbol(hb::hb_prof, z, sizeof(z));
    }
    return 0;
}
#endif

const char *hnsw_b200_last_error(void) { return hb::g_err.c_str(); }

const char *hnsw_b200_version(void) { return "hnsw_b200 0.2 sm_100a"; }

int32_t hnsw_b200_kernel_configs(int32_t dist_mode) {
    const int mode = dist_mode == HNSW_B200_DIST_BYTES
                         ? MODE_BYTES
                         : (dist_mode == HNSW_B200_DIST_EXACT_F32 ? MODE_EXACT : MODE_F64);
    return configs_of(mode);
}

const char *hnsw_b200_kernel_config_name(int32_t dist_mode, int32_t config) {
    if (config < 0 || config >= hnsw_b200_kernel_configs(dist_mode)) return "";
    return cfg_name(config);
}

int hnsw_b200_open(const hnsw_b200_graph_t *graph, void **handle) {
    if (!graph || !handle) return fail(HNSW_B200_EINVAL, "null argument");
    const hnsw_b200_graph_t &g = *graph;
    if (g.n <= 0 || g.n > 0x7ffffffe) return fail(HNSW_B200_EINVAL, "n must be in [1, 2^31 - 2]");
    if (g.dim <= 0) return fail(HNSW_B200_EINVAL, "dim must be positive");
    if (!g.vectors || !g.links0 || !g.count0 || !g.upper_offset)
        return fail(HNSW_B200_EINVAL, "graph arrays must be device pointers");
    if (g.metric < 0 || g.metric > 2) return fail(HNSW_B200_EINVAL, "unknown metric code");
    if (g.entry_point < 0 || g.entry_point >= g.n)
        return fail(HNSW_B200_EINVAL, "entry point outside the graph");
    if (g.max_level > 0 && (!g.links_up || !g.count_up || g.rows <= 0))
        return fail(HNSW_B200_EINVAL, "upper layers need links_up and count_up");
    Handle *h = new Handle();
    h->g = g;
    cudaGetDevice(&h->device);
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
    if (cudaMallocHost(reinterpret_cast<void **>(&h->host_pinned), 4 * sizeof(int32_t)) !=
        cudaSuccess) {
        delete h;
        return fail(HNSW_B200_ENOMEM, "pinned host allocation failed");
    }
    *handle = h;
    return 0;
}

void hnsw_b200_close(void *handle) {
    if (!handle) return;
    Handle *h = static_cast<Handle *>(handle);
    h->counters.release();
    h->status.release();
    h->qlist[0].release();
    h->qlist[1].release();
    h->order_rows.release();
    h->order_keys.release();
    h->order_list.release();
    h->sort_temp.release();
    h->vis.release();
    h->vbits.release();
    h->vlist.release();
    h->ties.release();
    h->spill_d.release();
    h->spill_i.release();
    h->spill_p.release();
    if (h->host_pinned) cudaFreeHost(h->host_pinned);
    delete h;
}

int64_t hnsw_b200_last_launches(void *handle) {
    return handle ? static_cast<Handle *>(handle)->launches : 0;
}

}  // extern "C"

namespace hb {

// The batched search. async = false: allocate scratch as needed, wait for the stream to read the
// overflow count and re-run overflowed queries with larger scratch. async = true: allocate nothing,
// synchronise nothing and read nothing on the host -- every launch goes on the stream (so a stream
// capture can record them); the scratch must already fit (a synchronous call with arguments of
// the same size sized it), and overflowed queries stay unwritten with their count left on the
// device for hnsw_b200_search_failed.
int search_impl(Handle &h, const hnsw_b200_search_args_t *a, cudaStream_t s, bool async) {
    h.launches = 0;
    const hnsw_b200_graph_t &g = h.g;
    if (a->nq < 0 || a->nq > 0x7fffffff) return fail(HNSW_B200_EINVAL, "nq out of range");
    if (a->nq == 0) return 0;
    if (a->k < 1 || a->k_search < a->k) return fail(HNSW_B200_EINVAL, "need 1 <= k <= k_search");
    if (!a->queries || !a->ef || !a->out_ids || !a->out_dists)
        return fail(HNSW_B200_EINVAL, "queries, ef and outputs must be device pointers");
    if (a->use_codes && !g.codes) return fail(HNSW_B200_EINVAL, "graph has no codes");
    if (a->dist_mode < HNSW_B200_DIST_F64 || a->dist_mode > HNSW_B200_DIST_BYTES)
        return fail(HNSW_B200_EINVAL, "unknown dist_mode");
    if (a->dist_mode != HNSW_B200_DIST_F64 && g.metric == HNSW_B200_COSINE)
        return fail(HNSW_B200_EINVAL, "exact integer modes need integer data (not cosine)");
    const uint8_t *rows8 = a->use_codes ? g.codes : g.vector_bytes;
    if (a->dist_mode == HNSW_B200_DIST_BYTES && (!rows8 || (g.dim & 3)))
        return fail(HNSW_B200_EINVAL, "byte mode needs uint8 rows and dim a multiple of 4");
    const bool filt = a->allowed != nullptr;
    const bool u8 = a->use_codes != 0;
    const int mode = a->dist_mode == HNSW_B200_DIST_BYTES
                         ? MODE_BYTES
                         : (a->dist_mode == HNSW_B200_DIST_EXACT_F32 ? MODE_EXACT : MODE_F64);
    const int ef_cap = std::max(std::max(a->ef_max, a->k_search), 1);
    const int krr = a->rerank_queries ? a->k : 0;
    const int s_cap = 256;
    const int cfg = a->kernel_config;
    if (cfg < 0 || cfg >= configs_of(mode))
        return fail(HNSW_B200_EINVAL, "kernel_config " + std::to_string(cfg) + " out of range (" +
                                          std::to_string(configs_of(mode)) + " for this mode)");
    // One lane per neighbour's row: a win unless the filter is very selective, where most rows it
    // would fetch early belong to neighbours already visited.
    const double p = filt ? std::max(double(a->allowed_fraction), 1.0 / double(g.n)) : 1.0;
    const int lane_rows = (!filt || p >= HB_LANE_ROWS_MIN_P) ? 1 : 0;
    const size_t wb = warp_smem_bytes(ef_cap, g.dim, filt, s_cap, krr, g.node_ids != nullptr,
                                      stage_bytes(mode, cfg, lane_rows, g.dim));
    const bool use_mlp = a->stop_mlp != nullptr && !filt;
    const size_t smem_block = wb * WPB + (use_mlp ? al16(MLP_BYTES) : 0);
    if (a->trace_feat && (!a->trace_dk || !a->trace_count || !a->trace_hops || a->trace_cap < 1))
        return fail(HNSW_B200_EINVAL, "trace needs trace_dk, trace_count, trace_hops and trace_cap");
    if (smem_block > 227 * 1024)
        return fail(HNSW_B200_EINVAL, "ef/dim too large for shared memory (" +
                                          std::to_string(smem_block) + " bytes per block)");
    int bps = 0;
    if (int rc = occupancy(mode, u8, filt, cfg, smem_block, &bps)) return rc;
    if (bps < 1) return fail(HNSW_B200_EINVAL, "search kernel cannot be resident");
    const int32_t nq = int32_t(a->nq);

    // Scratch sizing from the expected work per query: visits grow about linearly with ef and
    // inversely with the share of allowed nodes.
    const double est = std::min(double(g.n) + 64.0, (12.0 * ef_cap + 256.0) / p);
    int vis_log2 = std::max(8, ilog2_ceil(int64_t(2.0 * est)));
    int vis_up_log2 = 10;
    int tie_cap = ef_cap + 64;
    const int64_t vbits_stride = ((g.n + 31) / 32 + 3) / 4 * 4;
    const int vlist_cap = int(std::min<int64_t>(65536, std::max<int64_t>(256, g.n / 256)));
    int spill_cap = filt ? int(std::min(double(g.n) + 64.0, est)) : 0;

    // Scratch: grown (zero-filled where noted) by a synchronous call; an asynchronous call only
    // checks that what it needs is already there.
    auto need = [&](Buffer &b, size_t bytes, bool zero = false) -> int {
        if (!async) return b.ensure(bytes, zero, s);
        if (b.bytes >= bytes && b.ptr) return 0;
        return fail(HNSW_B200_EINVAL, "search_async: scratch for this batch is not reserved (run "
                                      "hnsw_b200_search once with arguments of this size first)");
    };
    if (int rc = need(h.counters, 4 * sizeof(int32_t))) return rc;
    if (int rc = need(h.status, size_t(nq) * sizeof(int32_t))) return rc;
    if (!async) {
        if (int rc = h.qlist[0].ensure(size_t(nq) * sizeof(int32_t))) return rc;
        if (int rc = h.qlist[1].ensure(size_t(nq) * sizeof(int32_t))) return rc;
    }
    int32_t *ctr = static_cast<int32_t *>(h.counters.ptr);

    SearchParams P;
    std::memset(&P, 0, sizeof(P));
    P.vectors = g.vectors;
    P.codes = g.codes;
    P.rows8 = rows8;
    P.links0 = g.links0;
    P.count0 = g.count0;
    P.upper_offset = g.upper_offset;
    P.links_up = g.links_up;
    P.count_up = g.count_up;
    P.n = g.n;
    P.node_ids = g.node_ids;
    P.dim = g.dim;
    P.links0_stride = g.links0_stride;
    P.links_up_stride = g.links_up_stride;
    P.metric = g.metric;
    P.entry_point = g.entry_point;
    P.max_level = g.max_level;
    P.queries = a->queries;
    P.queries_f64 = a->queries_f64;
    P.k = a->k;
    P.k_search = a->k_search;
    P.ef = a->ef;
    P.ef_cap = ef_cap;
    P.allowed = a->allowed;
    P.rerank_queries = a->rerank_queries;
    P.rerank_rows8 = (a->rerank_queries && g.vector_bytes && g.metric != HNSW_B200_COSINE &&
                      (g.dim & 15) == 0 && g.dim <= 128)
                         ? g.vector_bytes
                         : nullptr;
    P.out_ids = a->out_ids;
    P.out_dists = a->out_dists;
    P.out_ctr = a->out_counters;
    P.status = static_cast<int32_t *>(h.status.ptr);
    P.queue = ctr;
    P.n_failed = ctr + 1;
    P.s_cap = s_cap;
    P.stop_mlp = use_mlp ? a->stop_mlp : nullptr;
    P.stop_threshold = a->stop_threshold;
    P.stop_slope = a->stop_slope;
    P.stop_slope_from = a->stop_slope_from;
    P.trace_feat = filt ? nullptr : a->trace_feat;
    P.trace_dk = a->trace_dk;
    P.trace_count = a->trace_count;
    P.trace_hops = a->trace_hops;
    P.trace_cap = a->trace_cap;
    P.cells = a->cell_cost && a->n_cells > 0 ? a->cells : nullptr;
    P.cell_cost = a->cell_cost;
    P.n_cells = a->n_cells;
    P.trace_k = 16;
    P.lane_rows = lane_rows;

    int32_t n_work = nq;
    const int32_t *qlist = nullptr;
    if (a->priority && nq > 1) {
        // First work list: rows by descending priority, stably (CUB radix sort of the low 16 bits
        // of the keys with the rows as values); always a permutation of the rows.
        const size_t rb = size_t(nq) * sizeof(int32_t);
        if (int rc = need(h.order_rows, rb)) return rc;
        if (int rc = need(h.order_keys, rb)) return rc;
        if (int rc = need(h.order_list, rb)) return rc;
        int32_t *rows = static_cast<int32_t *>(h.order_rows.ptr);
        int32_t *keys = static_cast<int32_t *>(h.order_keys.ptr);
        int32_t *list = static_cast<int32_t *>(h.order_list.ptr);
        iota_rows<<<std::max(1, std::min(1024, (nq + 255) / 256)), 256, 0, s>>>(rows, nq);
        CUDA_TRY(cudaGetLastError());
        h.launches++;
        size_t temp = 0;
        CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(nullptr, temp, a->priority, keys, rows,
                                                           list, nq, 0, 16, s));
        if (int rc = need(h.sort_temp, std::max<size_t>(temp, 16))) return rc;
        CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(h.sort_temp.ptr, temp, a->priority, keys,
                                                           rows, list, nq, 0, 16, s));
        qlist = list;
    }
    for (int attempt = 0; attempt < 6; attempt++) {
        const int blocks = int(std::min<int64_t>(int64_t(h.sms) * bps, (n_work + WPB - 1) / WPB));
        const int64_t slots = int64_t(blocks) * WPB;
        // Unfiltered layer 0 uses the bitmap unless the configuration uses its hash.
        const int64_t vis_stride = int64_t(1) << (cfg_hash(cfg) && !filt ? std::max(vis_log2, vis_up_log2)
                                                                      : vis_up_log2);
        if (int rc = need(h.vis, size_t(slots * vis_stride) * sizeof(int32_t))) return rc;
        if (h.bits_dirty && h.vbits.ptr) {
            if (async) return fail(HNSW_B200_EINVAL, "search_async: a failed launch left the bitmaps "
                                                     "dirty; run hnsw_b200_search first");
            CUDA_TRY(cudaMemsetAsync(h.vbits.ptr, 0, h.vbits.bytes, s));
            h.bits_dirty = false;
        }
        if (int rc = need(h.vbits, size_t(slots * vbits_stride) * sizeof(uint32_t), true)) return rc;
        if (int rc = need(h.vlist, size_t(slots) * vlist_cap * sizeof(int32_t))) return rc;
        if (int rc = need(h.ties, size_t(slots) * tie_cap * sizeof(int32_t))) return rc;
        if (filt) {
            if (int rc = need(h.spill_d, size_t(slots) * spill_cap * sizeof(double))) return rc;
            if (int rc = need(h.spill_i, size_t(slots) * spill_cap * sizeof(int32_t))) return rc;
            if (g.node_ids)
                if (int rc = need(h.spill_p, size_t(slots) * spill_cap * sizeof(int32_t))) return rc;
        }
        P.vbits = static_cast<uint32_t *>(h.vbits.ptr);
        P.vbits_stride = vbits_stride;
        P.vlist = static_cast<int32_t *>(h.vlist.ptr);
        P.vlist_cap = vlist_cap;
        P.vis = static_cast<int32_t *>(h.vis.ptr);
        P.vis_stride = vis_stride;
        P.vis_log2 = vis_log2;
        P.vis_up_log2 = vis_up_log2;
        P.ties = static_cast<int32_t *>(h.ties.ptr);
        P.tie_cap = tie_cap;
        P.spill_d = static_cast<double *>(h.spill_d.ptr);
        P.spill_i = static_cast<int32_t *>(h.spill_i.ptr);
        P.spill_p = static_cast<int32_t *>(h.spill_p.ptr);
        P.spill_cap = spill_cap;
        P.qlist = qlist;
        P.n_work = n_work;
        CUDA_TRY(cudaMemsetAsync(ctr, 0, 4 * sizeof(int32_t), s));
        if (int rc = dispatch(P, mode, u8, filt, cfg, smem_block, blocks, s)) {
            h.bits_dirty = true;
            return rc;
        }
        h.launches++;
        if (async) return 0;  // the overflow count stays on the device
        CUDA_TRY(cudaMemcpyAsync(h.host_pinned, ctr, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            h.bits_dirty = true;
            return fail(HNSW_B200_ECUDA, std::string("search kernel failed: ") +
                                             cudaGetErrorString(cudaGetLastError()));
        }
        const int32_t failed = h.host_pinned[1];
        if (failed == 0) return 0;
        // Re-run the overflowed queries with four times the scratch of every kind.
        int32_t *list = static_cast<int32_t *>(h.qlist[attempt & 1].ptr);
        CUDA_TRY(cudaMemsetAsync(ctr + 2, 0, sizeof(int32_t), s));
        collect_failed<<<std::max(1, std::min(1024, (n_work + 255) / 256)), 256, 0, s>>>(
            P.status, qlist, n_work, list, ctr + 2);
        CUDA_TRY(cudaGetLastError());
        h.launches++;
        CUDA_TRY(cudaStreamSynchronize(s));
        n_work = failed;
        qlist = list;
        vis_log2 = std::min(vis_log2 + 2, ilog2_ceil(2 * g.n + 64));
        vis_up_log2 = std::min(vis_up_log2 + 2, ilog2_ceil(2 * g.n + 64));
        vis_log2 = std::max(vis_log2, 8);
        vis_up_log2 = std::max(vis_up_log2, 8);
        tie_cap *= 4;
        if (filt) spill_cap = int(std::min<int64_t>(int64_t(spill_cap) * 4, g.n + 64));
    }
    return fail(HNSW_B200_ERETRY, "queries still overflowed scratch after retries");
}

}  // namespace hb

extern "C" {

int hnsw_b200_search(void *handle, const hnsw_b200_search_args_t *a, void *stream) {
    if (!handle || !a) return fail(HNSW_B200_EINVAL, "null argument");
    Handle &h = *static_cast<Handle *>(handle);
    std::lock_guard<std::mutex> lock(h.mu);
    return search_impl(h, a, static_cast<cudaStream_t>(stream), false);
}

int hnsw_b200_search_async(void *handle, const hnsw_b200_search_args_t *a, void *stream) {
    if (!handle || !a) return fail(HNSW_B200_EINVAL, "null argument");
    Handle &h = *static_cast<Handle *>(handle);
    std::lock_guard<std::mutex> lock(h.mu);
    return search_impl(h, a, static_cast<cudaStream_t>(stream), true);
}

int hnsw_b200_search_failed(void *handle, int32_t *failed, void *stream) {
    if (!handle || !failed) return fail(HNSW_B200_EINVAL, "null argument");
    Handle &h = *static_cast<Handle *>(handle);
    std::lock_guard<std::mutex> lock(h.mu);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!h.counters.ptr) {
        *failed = 0;
        return 0;
    }
    CUDA_TRY(cudaMemcpyAsync(h.host_pinned, static_cast<int32_t *>(h.counters.ptr),
                             4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    *failed = h.host_pinned[1];
    return 0;
}

}  // extern "C"

// =========================================================================== fixed-scratch search
// Some callers cannot allocate device memory at all: real-time serving loops where an allocation
// would stall the loop, plugins whose host owns every device allocation through its own pool, and
// processes started under a hard device-memory budget. For them hnsw_b200_search_noalloc runs the
// same search kernel with all of its working memory carved out of one fixed array that is part of
// the library image. The array is HB_NOALLOC_BYTES (32 MiB) of device memory that every GPU which
// loads this library keeps until the process exits, whether or not the entry point is used. The
// call waits for its stream once before returning, to read how many queries overflowed.
namespace hb {

constexpr size_t HB_NOALLOC_BYTES = size_t(32) << 20;
constexpr int32_t HB_NOALLOC_MAX_NQ = 1 << 20;  // per-query status words live in the array too
static __device__ __align__(256) unsigned char g_noalloc_scratch[HB_NOALLOC_BYTES];

// Device address of g_noalloc_scratch on the current device. The host-side symbol is only a
// handle, not an address a kernel may use. It is looked up on every call rather than cached, so a
// context that was destroyed and recreated (cudaDeviceReset) never leaves a stale pointer behind.
int noalloc_scratch(void **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(HNSW_B200_ECUDA, std::string("search_noalloc: cudaGetSymbolAddress failed: ") +
                                         cudaGetErrorString(e));
    *out = p;
    return 0;
}

}  // namespace hb

extern "C" int hnsw_b200_search_noalloc(const hnsw_b200_graph_t *graph,
                                        const hnsw_b200_search_args_t *a, void *stream) {
    using namespace hb;
    if (!graph || !a) return fail(HNSW_B200_EINVAL, "null argument");
    const hnsw_b200_graph_t &g = *graph;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (g.n <= 0 || g.n > 0x7ffffffe || g.dim <= 0 || !g.vectors || !g.links0 || !g.count0 ||
        !g.upper_offset || g.entry_point < 0 || g.entry_point >= g.n || g.metric < 0 || g.metric > 2)
        return fail(HNSW_B200_EINVAL, "search_noalloc: invalid graph");
    if (g.max_level > 0 && (!g.links_up || !g.count_up || g.rows <= 0))
        return fail(HNSW_B200_EINVAL, "search_noalloc: upper layers need links_up and count_up");
    if (a->allowed) return fail(HNSW_B200_EINVAL, "search_noalloc: filtered search needs hnsw_b200_search");
    if (a->priority)
        return fail(HNSW_B200_EINVAL, "search_noalloc: no start order (priority must be NULL)");
    if (a->kernel_config != 0)
        return fail(HNSW_B200_EINVAL, "search_noalloc: runs kernel configuration 0 only");
    if (a->nq < 0) return fail(HNSW_B200_EINVAL, "nq out of range");
    if (a->nq > HB_NOALLOC_MAX_NQ)
        return fail(HNSW_B200_EINVAL, "search_noalloc: at most " + std::to_string(HB_NOALLOC_MAX_NQ) +
                                          " queries per call (split the batch)");
    if (a->nq == 0) return 0;
    if (a->k < 1 || a->k_search < a->k) return fail(HNSW_B200_EINVAL, "need 1 <= k <= k_search");
    if (!a->queries || !a->ef || !a->out_ids || !a->out_dists)
        return fail(HNSW_B200_EINVAL, "queries, ef and outputs must be device pointers");
    if (a->use_codes && !g.codes) return fail(HNSW_B200_EINVAL, "graph has no codes");
    if (a->dist_mode < HNSW_B200_DIST_F64 || a->dist_mode > HNSW_B200_DIST_BYTES)
        return fail(HNSW_B200_EINVAL, "unknown dist_mode");
    if (a->dist_mode != HNSW_B200_DIST_F64 && g.metric == HNSW_B200_COSINE)
        return fail(HNSW_B200_EINVAL, "exact integer modes need integer data (not cosine)");
    const uint8_t *rows8 = a->use_codes ? g.codes : g.vector_bytes;
    if (a->dist_mode == HNSW_B200_DIST_BYTES && (!rows8 || (g.dim & 3)))
        return fail(HNSW_B200_EINVAL, "byte mode needs uint8 rows and dim a multiple of 4");
    if (a->trace_feat && (!a->trace_dk || !a->trace_count || !a->trace_hops || a->trace_cap < 1))
        return fail(HNSW_B200_EINVAL, "trace needs trace_dk, trace_count, trace_hops and trace_cap");
    const bool u8 = a->use_codes != 0;
    const int mode = a->dist_mode == HNSW_B200_DIST_BYTES
                         ? MODE_BYTES
                         : (a->dist_mode == HNSW_B200_DIST_EXACT_F32 ? MODE_EXACT : MODE_F64);
    const int ef_cap = std::max(std::max(a->ef_max, a->k_search), 1);
    const int krr = a->rerank_queries ? a->k : 0;
    const size_t wb = warp_smem_bytes(ef_cap, g.dim, false, 256, krr, g.node_ids != nullptr,
                                      stage_bytes(mode, 0, 1, g.dim));
    const bool use_mlp = a->stop_mlp != nullptr;
    const size_t smem_block = wb * WPB + (use_mlp ? al16(MLP_BYTES) : 0);
    if (smem_block > 227 * 1024) return fail(HNSW_B200_EINVAL, "ef/dim too large for shared memory");
    // Carve the fixed array: counters, per-query status, then per warp slot the layer-0 bitmap, its
    // list of marked ids, the upper-layer hash and the tie stack. The slot count is whatever fits.
    // Requests that cannot fit are rejected here, before any CUDA call.
    const int32_t nq = int32_t(a->nq);
    const int64_t vbits_stride = ((g.n + 31) / 32 + 3) / 4 * 4;
    const int vlist_cap = int(std::min<int64_t>(65536, std::max<int64_t>(256, g.n / 256)));
    const int vis_up_log2 = 10;
    const int tie_cap = ef_cap + 64;
    const size_t head = al16(4 * sizeof(int32_t)) + al16(size_t(nq) * sizeof(int32_t));
    const size_t per_slot = size_t(vbits_stride) * 4 + al16(size_t(vlist_cap) * 4) +
                            (size_t(1) << vis_up_log2) * 4 + al16(size_t(tie_cap) * 4);
    if (head + per_slot * WPB > HB_NOALLOC_BYTES)
        return fail(HNSW_B200_EINVAL, "search_noalloc: graph of " + std::to_string(g.n) +
                                          " nodes needs more than the fixed " +
                                          std::to_string(HB_NOALLOC_BYTES >> 20) + " MiB scratch");
    int bps = 0;
    if (int rc = occupancy(mode, u8, false, 0, smem_block, &bps)) return rc;
    if (bps < 1) return fail(HNSW_B200_EINVAL, "search kernel cannot be resident");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void *base = nullptr;
    if (int rc = noalloc_scratch(&base)) return rc;
    const int64_t slot_fit = int64_t((HB_NOALLOC_BYTES - head) / per_slot) / WPB * WPB;
    const int blocks = int(std::min<int64_t>(std::min<int64_t>(int64_t(sms) * bps, slot_fit / WPB),
                                             (nq + WPB - 1) / WPB));
    const int64_t slots = int64_t(blocks) * WPB;
    unsigned char *p = static_cast<unsigned char *>(base);
    int32_t *ctr = reinterpret_cast<int32_t *>(p);
    int32_t *status = reinterpret_cast<int32_t *>(p + al16(4 * sizeof(int32_t)));
    unsigned char *q = p + head;
    uint32_t *vbits = reinterpret_cast<uint32_t *>(q);
    q += size_t(slots) * vbits_stride * 4;
    int32_t *vlist = reinterpret_cast<int32_t *>(q);
    q += al16(size_t(slots) * vlist_cap * 4);
    int32_t *vis = reinterpret_cast<int32_t *>(q);
    q += size_t(slots) << vis_up_log2 << 2;
    int32_t *ties = reinterpret_cast<int32_t *>(q);
    // The array keeps the previous call's contents: zero the counters and the bitmaps (each
    // query clears its own bits, but a previous call may have stopped part-way).
    CUDA_TRY(cudaMemsetAsync(ctr, 0, 4 * sizeof(int32_t), s));
    CUDA_TRY(cudaMemsetAsync(vbits, 0, size_t(slots) * vbits_stride * 4, s));

    SearchParams P;
    std::memset(&P, 0, sizeof(P));
    P.vectors = g.vectors;
    P.codes = g.codes;
    P.rows8 = rows8;
    P.links0 = g.links0;
    P.count0 = g.count0;
    P.upper_offset = g.upper_offset;
    P.links_up = g.links_up;
    P.count_up = g.count_up;
    P.n = g.n;
    P.node_ids = g.node_ids;
    P.dim = g.dim;
    P.links0_stride = g.links0_stride;
    P.links_up_stride = g.links_up_stride;
    P.metric = g.metric;
    P.entry_point = g.entry_point;
    P.max_level = g.max_level;
    P.queries = a->queries;
    P.queries_f64 = a->queries_f64;
    P.qlist = nullptr;
    P.n_work = nq;
    P.k = a->k;
    P.k_search = a->k_search;
    P.ef = a->ef;
    P.ef_cap = ef_cap;
    P.rerank_queries = a->rerank_queries;
    P.rerank_rows8 = (a->rerank_queries && g.vector_bytes && g.metric != HNSW_B200_COSINE &&
                      (g.dim & 15) == 0 && g.dim <= 128)
                         ? g.vector_bytes
                         : nullptr;
    P.out_ids = a->out_ids;
    P.out_dists = a->out_dists;
    P.out_ctr = a->out_counters;
    P.status = status;
    P.queue = ctr;
    P.n_failed = ctr + 1;
    P.vbits = vbits;
    P.vbits_stride = vbits_stride;
    P.vlist = vlist;
    P.vlist_cap = vlist_cap;
    P.vis = vis;
    P.vis_stride = int64_t(1) << vis_up_log2;
    P.vis_log2 = 0;
    P.vis_up_log2 = vis_up_log2;
    P.ties = ties;
    P.tie_cap = tie_cap;
    P.s_cap = 256;
    P.stop_mlp = use_mlp ? a->stop_mlp : nullptr;
    P.stop_threshold = a->stop_threshold;
    P.stop_slope = a->stop_slope;
    P.stop_slope_from = a->stop_slope_from;
    P.trace_feat = a->trace_feat;
    P.trace_dk = a->trace_dk;
    P.trace_count = a->trace_count;
    P.trace_hops = a->trace_hops;
    P.trace_cap = a->trace_cap;
    P.cells = a->cell_cost && a->n_cells > 0 ? a->cells : nullptr;
    P.cell_cost = a->cell_cost;
    P.n_cells = a->n_cells;
    P.trace_k = 16;
    P.lane_rows = 1;
    const int rc = dispatch(P, mode, u8, false, 0, smem_block, blocks, s);
    if (rc) return rc;
    int32_t failed = 0;  // pageable host copy: no pinned allocation either
    CUDA_TRY(cudaMemcpyAsync(&failed, ctr + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (failed)
        return fail(HNSW_B200_ERETRY, "search_noalloc: " + std::to_string(failed) +
                                          " queries overflowed the fixed scratch (their outputs are "
                                          "not written); search them with hnsw_b200_search");
    return 0;
}
