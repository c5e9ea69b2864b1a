// Exact brute-force k-NN on B200 tensor cores (the reference's oracle.exact_search,
// src/hnsw_engine/oracle.py:35-126, re-designed for sm_100a).
//
// Algorithm (the reference's filter-then-rerank, with this kernel's own error bound):
//  1. prep: rows -> BF16 operands. Integer data with |v| <= 256 is exact in BF16 (one term). Other
//     data is split v = hi + lo (hi = bf16(v), lo = bf16(v - hi)) and the operands are concatenated
//     along K as Q' = [q_hi, q_hi, q_lo], X' = [x_hi, x_lo, x_hi], so one GEMM yields
//     hi.hi + hi.lo + lo.hi (relative error about 2^-16). Norms are computed in float64.
//  2. filter GEMM (tcgen05.mma kind::f16, BF16 x BF16 -> FP32 in TMEM, TMA-fed, warp specialised):
//     approx distance a = |q|^2 + |x|^2 - 2 q.x (l2), -q.x (ip) or 1 - q.x (cosine, on float64-
//     normalised rows); every (query, row) with a <= tau_q + margin_q is appended to the query's
//     candidate list. margin_q = 2 e_q where e_q bounds |a - exact| for this arithmetic, so every true
//     top-k row survives whenever tau_q is at least the k-th smallest approximate distance.
//  3. tau_q: pass one runs the filter on a prefix of the data with tau = +inf, and a radix select
//     takes the k-th smallest approximate distance of that prefix (an upper bound of the global one).
//     Pass two filters all rows; a second select tightens tau to the k-th smallest candidate.
//  4. rerank: float64 distances (sequential over dimensions) of the surviving candidates, best k by
//     (distance, id) -- ties to the lower id, as np.lexsort((ids, exact)) in the reference.
// Waits on mbarriers are bounded by a wall-clock limit; on expiry the kernel records an error,
// drains what it issued and frees its TMEM.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "hnsw_b200.h"

namespace hb {
int fail(int code, const std::string &msg);  // search.cu: records the thread's last error
}

namespace hbx {

constexpr int BM = 128;  // queries per tile (TMEM lanes)
constexpr int BN = 256;  // data rows per tile (TMEM columns per accumulator)
constexpr int BK = 64;   // K elements per stage (128 bytes of BF16: one swizzle-128B row)
constexpr int STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;
constexpr int B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
// Epilogue warps: EPI_WARPS / 4 per TMEM lane quarter, taking a tile's CW-column chunks in turn.
// Narrower chunks need fewer registers per thread, which leaves room for more epilogue warps to
// hide the TMEM-load and arithmetic latencies.
#ifndef HB_EPI_WARPS
#define HB_EPI_WARPS 20
#endif
#ifndef HB_EPI_CW
#define HB_EPI_CW 16
#endif
constexpr int EPI_WARPS = HB_EPI_WARPS;
constexpr int CW = HB_EPI_CW;  // columns per TMEM load (16 or 32)
static_assert(CW == 16 || CW == 32, "chunks of 16 or 32 columns");
constexpr int EPI_PER_QUARTER = EPI_WARPS / 4;
constexpr int FILTER_THREADS = 128 + 32 * EPI_WARPS;
constexpr int BAR_BYTES = 256;  // barriers and flags after the stage buffers and the |x|^2 ring
constexpr int XSLOTS = 4;       // |x|^2 ring slots (one tile's BN values each)
// Rows of at least COOP_DIM dimensions are re-scored by the whole warp, one candidate at a time.
constexpr int COOP_DIM = 256;
// Byte rows: one result in VERIFY_EVERY of each query is re-scored in float64 as a check.
constexpr int VERIFY_EVERY = 16;
constexpr uint32_t TMEM_COLS = 512;  // two accumulators of BN columns
constexpr unsigned long long WAIT_LIMIT_NS = 4000000000ull;  // 4 s

// UMMA instruction descriptor: BF16 A and B (K-major), FP32 accumulator, M = 128, N = 256.
constexpr uint32_t IDESC = (1u << 4)            // c_format F32
                           | (1u << 7)          // a_format BF16
                           | (1u << 10)         // b_format BF16
                           | (uint32_t(BN >> 3) << 17) | (uint32_t(BM >> 4) << 24);
// The same for byte rows (kind::i8): unsigned 8-bit A and B (formats 0), S32 accumulator (c_format
// 2). Integer products and sums are exact, so the filter values are the exact distances.
constexpr uint32_t IDESC_I8 = (2u << 4) | (uint32_t(BN >> 3) << 17) | (uint32_t(BM >> 4) << 24);
// Byte rows: a K chunk of one stage is 128 elements (one 128-byte swizzle row), 32 per instruction.
constexpr int BK8 = 128;
// Largest |distance| whose float value is exact (integers below 2^24).
constexpr float EXACT_LIM = 16777216.f;
// Filter value of a padding column in the byte path: above every distance the path admits.
constexpr int32_t I8_PAD = 0x3fffffff;

struct FilterParams {
    int32_t nq;            // valid queries
    int32_t row_begin;     // first data row of this pass
    int32_t row_end;       // one past the last data row of this pass
    int32_t kchunks;       // K' / BK
    int32_t tiles_per_split;
    int32_t metric;
    const float *qq;       // |q|^2 per query (l2)
    const float *xx;       // |x|^2 per row (l2)
    const int32_t *qqi;    // byte rows: exact |q|^2 per query (l2)
    const int32_t *xxi;    // byte rows: exact |x|^2 per row (l2)
    const float *thr;      // per query: tau + margin (+inf in pass one)
    // Candidates in segments: every epilogue thread of the grid owns one segment of its query's
    // list (segment = row split x epilogue part), so appends need no atomics. Segment s of query q
    // starts at (q * nseg + s) * cap.
    float *cand_val;       // (nq, nseg, cap) approximate distances
    int32_t *cand_id;      // (nq, nseg, cap) row ids
    int32_t *cand_cnt;     // (nq, nseg) appended counts (may exceed cap: overflow)
    int32_t cap;           // entries per segment
    int32_t block_min;     // 1: append only the minimum of each (tile, part) block (threshold pass)
    int32_t *err;          // nonzero: a bounded wait expired
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One bounded probe of a barrier phase. The thread may be suspended by the hardware for up to
// MBAR_SUSPEND_NS while the phase is incomplete (instead of spinning on issue slots).
constexpr uint32_t MBAR_SUSPEND_NS = 100000;  // 0.1 ms
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(MBAR_SUSPEND_NS)
        : "memory");
    return ok != 0;
}

// Bounded wait: false if the wall-clock limit expired (the caller records the error).
// The abort flag and the clock are read every 64th probe: a waiting thread then issues little
// besides the probes, leaving the issue slots to the warps that work.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (uint32_t i = 1;; i++) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 63u) == 0u) {
            if (*abort_flag) return false;
            if (now_ns() - t0 > WAIT_LIMIT_NS) return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap *map, uint64_t *bar, void *dst, int x,
                                            int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Plain (untiled, non-multicast) bulk copy of `bytes` from this GPU's global memory into shared
// memory, completing on bar: both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor, K-major, 128-byte swizzle: rows of 128 bytes, 8-row groups
// 1024 bytes apart (stride byte offset), leading byte offset 16 bytes, descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFF);
    d |= uint64_t(1) << 16;            // leading byte offset (16 B) >> 4
    d |= uint64_t(1024 >> 4) << 32;    // stride byte offset >> 4
    d |= uint64_t(1) << 46;            // version
    d |= uint64_t(2) << 61;            // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_u8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(IDESC_I8), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

template <int W>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[W]) {
    if constexpr (W == 16) tmem_ld16(taddr, v);
    else tmem_ld32(taddr, v);
}

// I8: byte rows on kind::i8 (exact integer filter values); otherwise BF16 terms on kind::f16.
template <bool I8>
__global__ void __launch_bounds__(FILTER_THREADS, 1)
    knn_filter_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const FilterParams p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned stage buffers (swizzle-128B atoms), barriers after them.
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    // |x|^2 of a tile's BN rows (float or int32, 4 bytes each) in a ring of XSLOTS, after the
    // stages: the producer fills slot lt % XSLOTS, the epilogue reads it and releases it.
    unsigned char *xring = smem + STAGES * STAGE_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(xring + XSLOTS * BN * 4);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *xfull = tempty + 2;
    uint64_t *xempty = xfull + XSLOTS;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(xempty + XSLOTS);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int qt = blockIdx.x;
    const int total_tiles = (p.row_end - p.row_begin + BN - 1) / BN;
    const int t0 = blockIdx.y * p.tiles_per_split;
    const int t1 = min(total_tiles, t0 + p.tiles_per_split);
    const int ntiles = max(0, t1 - t0);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(tfull + b, 1);
            mbar_init(tempty + b, EPI_WARPS);
        }
        for (int x = 0; x < XSLOTS; x++) {
            mbar_init(xfull + x, 1);
            mbar_init(xempty + x, EPI_WARPS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---------------------------------------------------------------- TMA producer
        int it = 0, xs = 0;  // stages and |x|^2 slots issued
        bool ok = true;
        for (int lt = 0; lt < ntiles && ok; lt++) {
            const int row0 = p.row_begin + (t0 + lt) * BN;
            {  // the tile's |x|^2 (rows row0 .. row0 + BN - 1 < n_pad) into its ring slot
                const int x = lt % XSLOTS;
                if (!mbar_wait(xempty + x, ((lt / XSLOTS) & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(xfull + x, BN * 4);
                const void *src = I8 ? static_cast<const void *>(p.xxi + row0)
                                     : static_cast<const void *>(p.xx + row0);
                bulk_load(xring + x * BN * 4, src, BN * 4, xfull + x);
                xs++;
            }
            for (int kc = 0; kc < p.kchunks; kc++, it++) {
                const int s = it % STAGES;
                const uint32_t par = ((it / STAGES) & 1) ^ 1;
                if (!mbar_wait(empty + s, par, abort_flag)) {
                    ok = false;
                    break;
                }
                unsigned char *a = smem + s * STAGE_BYTES;
                unsigned char *b = a + A_BYTES;
                mbar_expect_tx(full + s, STAGE_BYTES);
                tma_load_2d(&tmA, full + s, a, kc * (I8 ? BK8 : BK), qt * BM);
                tma_load_2d(&tmB, full + s, b, kc * (I8 ? BK8 : BK), row0);
            }
        }
        if (!ok) {
            atomicExch(p.err, 1);
            *abort_flag = 1;
        }
        // Drain: every stage and |x|^2 slot issued must land before the CTA may exit.
        const int issued = it;
        for (int j = max(0, issued - STAGES); j < issued; j++) {
            const int s = j % STAGES;
            const uint32_t par = (j / STAGES) & 1;
            const unsigned long long t = now_ns();
            while (!mbar_try(full + s, par) && now_ns() - t < WAIT_LIMIT_NS) {
            }
        }
        for (int j = max(0, xs - XSLOTS); j < xs; j++) {
            const int x = j % XSLOTS;
            const uint32_t par = (j / XSLOTS) & 1;
            const unsigned long long t = now_ns();
            while (!mbar_try(xfull + x, par) && now_ns() - t < WAIT_LIMIT_NS) {
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------------------------------------------------------- MMA issuer
        int it = 0;
        bool ok = true;
        for (int lt = 0; lt < ntiles && ok; lt++) {
            const int b = lt & 1;
            if (!mbar_wait(tempty + b, ((lt >> 1) & 1) ^ 1, abort_flag)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t tmem_d = tmem_base + uint32_t(b * BN);
            for (int kc = 0; kc < p.kchunks; kc++, it++) {
                const int s = it % STAGES;
                if (!mbar_wait(full + s, (it / STAGES) & 1, abort_flag)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_addr = smem_u32(smem + s * STAGE_BYTES);
                const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
                for (int j = 0; j < 4; j++) {  // 32 bytes of K per instruction (16 BF16 or 32 bytes)
                    if constexpr (I8)
                        umma_u8(tmem_d, sw128_desc(a_addr + j * 32), sw128_desc(b_addr + j * 32),
                                (kc | j) != 0);
                    else
                        umma_bf16(tmem_d, sw128_desc(a_addr + j * 32), sw128_desc(b_addr + j * 32),
                                  (kc | j) != 0);
                }
                umma_commit(empty + s);
            }
            if (ok) umma_commit(tfull + b);
        }
        if (!ok) {
            atomicExch(p.err, 1);
            *abort_flag = 1;
        }
        // Every MMA issued must finish before TMEM is released: commit one more arrival on a
        // stage barrier and wait for it (tcgen05.commit tracks all prior MMAs of this thread).
        if (it > 0) {
            const int s = (it - 1) % STAGES;
            const uint32_t par = ((it - 1) / STAGES) & 1;
            const unsigned long long t = now_ns();
            while (!mbar_try(empty + s, par) && now_ns() - t < WAIT_LIMIT_NS) {
            }
        }
    } else if (warp >= 4) {
        // ---------------------------------------------------------------- epilogue
        // Warp w reads TMEM lanes 32 (w % 4) .. +31 (its hardware lane quarter: one query per
        // thread) and every EPI_PER_QUARTER-th 32-column chunk of each accumulator.
        const int quarter = warp & 3;
        const int part = (warp - 4) >> 2;  // 0 .. EPI_PER_QUARTER - 1
        const int row = quarter * 32 + lane;  // TMEM lane = query row of the tile
        const int q = qt * BM + row;
        const bool qvalid = q < p.nq;
        const float qq = (qvalid && !I8) ? p.qq[q] : 0.f;
        const int32_t qqi = (qvalid && I8) ? p.qqi[q] : 0;
        const float thr = qvalid ? p.thr[q] : -INFINITY;
        const int nseg = int(gridDim.y) * EPI_PER_QUARTER;
        const int64_t seg = int64_t(qvalid ? q : 0) * nseg + int64_t(blockIdx.y) * EPI_PER_QUARTER + part;
        float *cv = p.cand_val + seg * p.cap;
        int32_t *ci = p.cand_id + seg * p.cap;
        int cnt = 0;  // this thread's appends (its own segment: no atomics)
        const bool l2 = p.metric == HNSW_B200_L2;
        const bool cosine = p.metric == HNSW_B200_COSINE;
        for (int lt = 0; lt < ntiles; lt++) {
            const int b = lt & 1;
            const int row0 = p.row_begin + (t0 + lt) * BN;
            int ok = 1;
            if (lane == 0)
                ok = (mbar_wait(tfull + b, (lt >> 1) & 1, abort_flag) &&
                      mbar_wait(xfull + lt % XSLOTS, (lt / XSLOTS) & 1, abort_flag))
                         ? 1
                         : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0) {
                    atomicExch(p.err, 1);
                    *abort_flag = 1;
                }
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // TMEM columns of this warp's lane quarter in accumulator b; the tile's |x|^2 in its slot
            const uint32_t tbase = tmem_base + (uint32_t(quarter * 32) << 16) + uint32_t(b * BN);
            const unsigned char *xslot = xring + (lt % XSLOTS) * BN * 4;
            float tmin = INFINITY;  // threshold pass: minimum over this thread's chunks of the tile
            bool tany = false;
#pragma unroll 1
            for (int c = part * CW; c < BN; c += CW * EPI_PER_QUARTER) {
                const int col0 = row0 + c;
                const int valid = min(CW, p.row_end - col0);  // columns that are data rows
                // The filter value is a = v + vadd with v = |x|^2 - 2 q.x (l2), -q.x (ip, cosine)
                // and vadd = |q|^2, 0, 1: one FMA (integer multiply-add) or negation per element,
                // then the chunk's minimum. a is monotonic in v (float rounding included), so a
                // chunk whose minimum fails the threshold has no candidate; the rare chunks with
                // one test each element. |x|^2 of the CW columns comes from the tile's ring slot,
                // which the producer filled with one bulk copy (zero beyond the data rows): the
                // same addresses in every lane (shared-memory broadcasts) instead of an L2 round
                // trip per chunk (the whole 1M x 128 call: 6.95 against 7.06 ms).
                float v[CW];     // BF16 path: v; byte path: the raw S32 accumulator bits
                int32_t w[CW];   // byte path: v, exact
                float amin, vadd = 0.f;
                int32_t vaddi = 0;
                if constexpr (I8) {
                    int32_t xv[CW];
                    if (l2) {
                        const int4 *x4 = reinterpret_cast<const int4 *>(xslot) + c / 4;
#pragma unroll
                        for (int i = 0; i < CW / 4; i++) {
                            const int4 t = x4[i];
                            xv[4 * i] = t.x;
                            xv[4 * i + 1] = t.y;
                            xv[4 * i + 2] = t.z;
                            xv[4 * i + 3] = t.w;
                        }
                    }
                    tmem_ld<CW>(tbase + uint32_t(c), v);
#pragma unroll
                    for (int j = 0; j < CW; j++)
                        w[j] = l2 ? xv[j] - 2 * __float_as_int(v[j]) : -__float_as_int(v[j]);
                    if (valid < CW) {  // uniform: only the last tile of the rows
#pragma unroll
                        for (int j = 0; j < CW; j++)
                            if (j >= valid) w[j] = I8_PAD;
                    }
                    int32_t mh[CW / 2];
#pragma unroll
                    for (int j = 0; j < CW / 2; j++) mh[j] = min(w[j], w[j + CW / 2]);
#pragma unroll
                    for (int s2 = CW / 4; s2 > 0; s2 >>= 1)
#pragma unroll
                        for (int j = 0; j < s2; j++) mh[j] = min(mh[j], mh[j + s2]);
                    vaddi = l2 ? qqi : 0;
                    amin = float(mh[0] + vaddi);
                } else {
                    float xv[CW];
                    if (l2) {
                        const float4 *x4 = reinterpret_cast<const float4 *>(xslot) + c / 4;
#pragma unroll
                        for (int i = 0; i < CW / 4; i++) {
                            const float4 t = x4[i];
                            xv[4 * i] = t.x;
                            xv[4 * i + 1] = t.y;
                            xv[4 * i + 2] = t.z;
                            xv[4 * i + 3] = t.w;
                        }
                    }
                    tmem_ld<CW>(tbase + uint32_t(c), v);
                    if (l2) {
#pragma unroll
                        for (int j = 0; j < CW; j++) v[j] = fmaf(-2.f, v[j], xv[j]);
                    } else {
#pragma unroll
                        for (int j = 0; j < CW; j++) v[j] = -v[j];
                    }
                    if (valid < CW) {  // uniform: only the last tile of the rows
#pragma unroll
                        for (int j = 0; j < CW; j++)
                            if (j >= valid) v[j] = INFINITY;
                    }
                    float mh[CW / 2];
#pragma unroll
                    for (int j = 0; j < CW / 2; j++) mh[j] = fminf(v[j], v[j + CW / 2]);
#pragma unroll
                    for (int s2 = CW / 4; s2 > 0; s2 >>= 1)
#pragma unroll
                        for (int j = 0; j < s2; j++) mh[j] = fminf(mh[j], mh[j + s2]);
                    vadd = l2 ? qq : (cosine ? 1.f : 0.f);
                    amin = mh[0] + vadd;
                }
                if (p.block_min) {
                    if (valid > 0) {
                        tmin = fminf(tmin, amin);
                        tany = true;
                    }
                } else if (qvalid && amin <= thr) {
#pragma unroll
                    for (int j = 0; j < CW; j++) {  // static indices keep v[] in registers
                        const float a = I8 ? float(w[j] + vaddi) : v[j] + vadd;
                        if (j < valid && a <= thr) {
                            if (cnt < p.cap) {
                                cv[cnt] = a;
                                ci[cnt] = col0 + j;
                            }
                            cnt++;
                        }
                    }
                }
            }
            // Threshold pass: one value per (tile, part) block, the block's minimum. The k-th
            // smallest of the blocks' minima is at least the k-th smallest of all the values (a
            // subset's k-th is never below the set's), so it still bounds the k-th distance from
            // above; with far more blocks than k it is nearly as tight. Values only: the pass needs
            // no row ids.
            if (p.block_min && tany && qvalid) {
                if (cnt < p.cap) cv[cnt] = tmin;
                cnt++;
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(tempty + b);
                mbar_arrive(xempty + lt % XSLOTS);
            }
        }
        if (qvalid) p.cand_cnt[seg] = cnt;
    }
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(TMEM_COLS));
    }
}

// ------------------------------------------------------------------------------------- prep
// Byte rows (values checked to be integers in [0, 255]): one warp per row writes the u8 operand row
// of width kpad (a multiple of 128, zero past dim), four bytes a lane, and the exact |x|^2.
template <typename T>
__global__ void prep_rows_u8(const T *src, int64_t rows, int dim, int64_t rows_pad, int kpad,
                             uint8_t *dst, int32_t *sq) {
    const int lane = threadIdx.x & 31;
    const int64_t wpb = blockDim.x >> 5;
    for (int64_t r = int64_t(blockIdx.x) * wpb + (threadIdx.x >> 5); r < rows_pad;
         r += int64_t(gridDim.x) * wpb) {
        uint32_t *out = reinterpret_cast<uint32_t *>(dst + r * kpad);
        const T *x = src + r * dim;
        int32_t ss = 0;
        for (int i = lane * 4; i < kpad; i += 128) {
            uint32_t word = 0;
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int32_t v = (r < rows && i + t < dim) ? int32_t(x[i + t]) : 0;
                ss += v * v;
                word |= uint32_t(v & 255) << (8 * t);
            }
            out[i >> 2] = word;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        if (lane == 0) sq[r] = ss;
    }
}

// One warp per row: float64 norm, cosine normalisation, BF16 operand row(s) of width kpad.
// terms == 1: [v]; terms == 3: A-side [hi, hi, lo] (queries) or B-side [hi, lo, hi] (data).
template <typename T>
__global__ void prep_rows(const T *src, int64_t rows, int dim, int64_t rows_pad, int kpad,
                          int terms, int a_side, int cosine, __nv_bfloat16 *dst, double *norm64,
                          float *sq32) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int seg = kpad / terms;  // padded dim per term
    for (int64_t r = warp; r < rows_pad; r += nwarps) {
        __nv_bfloat16 *out = dst + r * kpad;
        if (r >= rows) {
            for (int i = lane; i < kpad; i += 32) out[i] = __float2bfloat16(0.f);
            if (lane == 0) {
                norm64[r] = 0.0;
                sq32[r] = 0.f;
            }
            continue;
        }
        const T *x = src + r * dim;
        double ss = 0.0;
        for (int i = lane; i < dim; i += 32) {
            const double v = double(x[i]);
            ss += v * v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        const double nrm = sqrt(ss);
        const double scale = cosine ? (nrm > 0 ? 1.0 / nrm : 0.0) : 1.0;
        for (int i = lane; i < seg; i += 32) {
            const double v = i < dim ? double(x[i]) * scale : 0.0;
            const float vf = float(v);
            const __nv_bfloat16 hi = __float2bfloat16_rn(vf);
            if (terms == 1) {
                out[i] = hi;
            } else {
                const __nv_bfloat16 lo = __float2bfloat16_rn(float(v - double(__bfloat162float(hi))));
                out[i] = hi;
                out[seg + i] = a_side ? hi : lo;
                out[2 * seg + i] = a_side ? lo : hi;
            }
        }
        if (lane == 0) {
            norm64[r] = nrm;  // cosine rerank re-normalises with it; margins use 1 for cosine
            sq32[r] = cosine ? 1.f : float(ss);
        }
    }
}

// ------------------------------------------------------------------------------ radix select
// Order-preserving key of a float (ascending floats -> ascending unsigned keys).
__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funkey(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Moves one query's candidates (segments of `cap` entries, counts in cnt) to the front of its
// region, in segment order, by one warp; returns how many there are. In place: an entry's new index
// (its rank in segment order) is never above its old one, and the warp moves the entries in rank
// order, 32 at a time, reading a batch before writing it, so no entry is overwritten before it has
// moved. A lane finds its entry's segment by a binary search over the 32 segment offsets of the
// group (shuffles).
__device__ __forceinline__ int compact_list(float *v, int32_t *id, const int32_t *cnt, int32_t cap,
                                            int32_t nseg, int lane) {
    int base = 0;
    for (int s0 = 0; s0 < nseg; s0 += 32) {
        const int sg = s0 + lane;
        const int n_sg = sg < nseg ? min(cnt[sg], cap) : 0;
        int incl = n_sg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - n_sg;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int b = 0; b < total; b += 32) {
            const int r = b + lane;  // rank within the group
            int lo = 0;  // last segment of the group whose offset is <= r (every lane searches)
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int e = __shfl_sync(0xffffffffu, excl, min(lo + step, 31));
                if (lo + step < 32 && e <= r) lo += step;
            }
            const int off = __shfl_sync(0xffffffffu, excl, lo);
            float val = 0.f;
            int32_t ident = 0;
            if (r < total) {
                const int64_t src = int64_t(s0 + lo) * cap + (r - off);
                val = v[src];
                if (id) ident = id[src];
            }
            __syncwarp();
            if (r < total) {
                v[base + r] = val;
                if (id) id[base + r] = ident;
            }
            __syncwarp();
        }
        base += total;
    }
    return base;
}

// One warp per query, 8 per block: tau[q] = k-th smallest of the candidate values (or +inf if
// fewer than k), then out_thr[q] = tau + margin[q]. A 4-pass radix select, 8 bits a pass, over the
// query's segments; the bin of the rank-th key comes from each lane's 8 bins and a warp scan.
constexpr int SELECT_WARPS = 8;
// The query's list is first compacted in place (compact_list) and its length stored in
// cand_m[q], so the radix passes and the re-rank read one dense run of entries.
__global__ void select_kth(float *cand_val, int32_t *cand_id, const int32_t *cand_cnt, int32_t cap,
                           int32_t nseg, int32_t nq, int32_t k, const float *margin, float *out_thr,
                           float *out_tau, int32_t *cand_m) {
    __shared__ uint32_t hist_all[SELECT_WARPS][256];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * SELECT_WARPS + wid;
    if (q >= nq) return;  // no block-wide barrier below
    uint32_t *hist = hist_all[wid];
    float *v = cand_val + int64_t(q) * nseg * cap;
    const int m = compact_list(v, cand_id ? cand_id + int64_t(q) * nseg * cap : nullptr,
                               cand_cnt + int64_t(q) * nseg, cap, nseg, lane);
    if (lane == 0) cand_m[q] = m;
    if (m < k) {
        if (lane == 0) {
            out_tau[q] = INFINITY;
            out_thr[q] = INFINITY;
        }
        return;
    }
    uint32_t prefix = 0, rank = uint32_t(k);  // rank: 1-based position within the current bucket
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = lane; i < 256; i += 32) hist[i] = 0;
        __syncwarp();
        const uint32_t hmask = shift == 24 ? 0u : (0xffffffffu << (shift + 8));
        for (int i = lane; i < m; i += 32) {
            const uint32_t key = fkey(v[i]);
            if ((key & hmask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncwarp();
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int b = 0; b < 8; b++) {
            c[b] = hist[lane * 8 + b];
            sum += c[b];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        uint32_t run = incl - sum, bucket = 0, nrank = 0;
        const bool mine = run < rank && rank <= incl;  // exactly one lane
        if (mine) {
#pragma unroll
            for (int b = 0; b < 8; b++) {
                if (nrank == 0 && run + c[b] >= rank) {
                    bucket = uint32_t(lane * 8 + b);
                    nrank = rank - run;
                }
                run += c[b];
            }
        }
        const int src = __ffs(__ballot_sync(0xffffffffu, mine)) - 1;
        bucket = __shfl_sync(0xffffffffu, bucket, src);
        nrank = __shfl_sync(0xffffffffu, nrank, src);
        prefix |= bucket << shift;
        rank = nrank;
        __syncwarp();
    }
    if (lane == 0) {
        const float tau = funkey(prefix);
        out_tau[q] = tau;
        out_thr[q] = tau + margin[q];
    }
}

// ------------------------------------------------------------------------------------ rerank
__device__ __forceinline__ bool pair_lt(double da, int32_t ia, double db, int32_t ib) {
    return da < db || (da == db && ia < ib);
}

// Float64 distance of row x to the query qv by one lane, the sums in dimension order.
template <typename T>
__device__ __forceinline__ double dist_f64_lane(const T *x, const T *qv, int dim, int metric,
                                                double xn, double qn) {
    double acc = 0.0;
    if (metric == HNSW_B200_L2) {
        for (int j = 0; j < dim; j++) {
            const double df = __dsub_rn(double(x[j]), double(qv[j]));
            acc = __dadd_rn(acc, __dmul_rn(df, df));
        }
        return acc;
    }
    if (metric == HNSW_B200_IP) {
        for (int j = 0; j < dim; j++) acc = __dadd_rn(acc, __dmul_rn(double(x[j]), double(qv[j])));
        return -acc;
    }
    for (int j = 0; j < dim; j++)
        acc = __dadd_rn(acc, __dmul_rn(__ddiv_rn(double(x[j]), xn), __ddiv_rn(double(qv[j]), qn)));
    return __dsub_rn(1.0, acc);
}

// The same by the whole warp (long rows): lane l sums dimensions l, l + 32, ..., then a fixed
// shuffle tree adds the lanes (the same value on every run; on integer data every order gives the
// same exact sum), so the float64 chains are 32 times shorter. The result is on every lane.
template <typename T>
__device__ __forceinline__ double dist_f64_warp(const T *x, const T *qv, int dim, int metric,
                                                double xn, double qn, int lane) {
    double acc = 0.0;
    if (metric == HNSW_B200_L2) {
        for (int i = lane; i < dim; i += 32) {
            const double df = __dsub_rn(double(x[i]), double(qv[i]));
            acc = __dadd_rn(acc, __dmul_rn(df, df));
        }
    } else if (metric == HNSW_B200_IP) {
        for (int i = lane; i < dim; i += 32) acc = __dadd_rn(acc, __dmul_rn(double(x[i]), double(qv[i])));
    } else {
        for (int i = lane; i < dim; i += 32)
            acc = __dadd_rn(acc, __dmul_rn(__ddiv_rn(double(x[i]), xn), __ddiv_rn(double(qv[i]), qn)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
    return metric == HNSW_B200_L2 ? acc : (metric == HNSW_B200_IP ? -acc : __dsub_rn(1.0, acc));
}

// One warp per query: exact float64 distances of the candidates within the final threshold,
// best k by (distance, id) kept in shared memory (sorted insertion), written as int64 / float64.
// exact_lim > 0 (byte rows, integer filter): a candidate whose filter value is below exact_lim in
// magnitude already holds its exact distance and is not re-scored; one result in VERIFY_EVERY of
// every query (positions q, q + VERIFY_EVERY, ... mod VERIFY_EVERY, so a batch covers every
// position) is re-scored in float64 at the end instead, and any difference sets *mismatch. (Re-scoring every query's results cost 0.55 ms of 8.6 on the 1M x 128 mixture and
// 0.63 of 2.6 on the 60K x 784 set, 10K queries each; integer products and sums are exact, so
// the check is there to catch a wrong operand layout or descriptor, which a sample shows.)
template <typename T>
__global__ void rerank_topk(const T *data, const T *queries, int dim, int32_t nq, int32_t k,
                            int32_t metric, const double *xnorm, const double *qnorm,
                            const float *cand_val, const int32_t *cand_id, const int32_t *cand_m,
                            int32_t cap, int32_t nseg, const float *thr, int64_t *out_ids,
                            double *out_d, unsigned long long *err_max, float exact_lim,
                            int32_t *mismatch) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int warps = blockDim.x >> 5;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x * warps + w;
    double *Ad = reinterpret_cast<double *>(sm) + size_t(w) * (k + 1);
    int32_t *Ai = reinterpret_cast<int32_t *>(reinterpret_cast<double *>(sm) + size_t(warps) * (k + 1)) +
                  size_t(w) * (k + 1);
    if (q >= nq) return;
    const float t = thr[q];
    const T *qv = queries + int64_t(q) * dim;
    const bool cos = metric == HNSW_B200_COSINE;
    const double qn = cos ? qnorm[q] : 1.0;
    int a = 0;
    double err = 0.0;  // largest |filter value - exact distance| over this lane's re-scored survivors
    // The query's candidates, compacted by select_kth to the front of its region: batches of 32,
    // one per lane.
    const int m = cand_m[q];
    const int64_t region = int64_t(q) * nseg * cap;
    for (int b0 = 0; b0 < m; b0 += 32) {
        const int64_t at = b0 + lane < m ? region + b0 + lane : -1;  // this lane's entry
        const float approx = at >= 0 ? cand_val[at] : INFINITY;
        const bool has = at >= 0 && approx <= t;
        const int32_t id = has ? cand_id[at] : -1;
        const bool known = has && fabsf(approx) < exact_lim;  // exact already (byte rows)
        const bool need = has && !known;
        double d = known ? double(approx) : INFINITY;
        if (dim >= COOP_DIM) {
            for (uint32_t hm = __ballot_sync(0xffffffffu, need); hm; hm &= hm - 1) {
                const int j = __ffs(hm) - 1;
                const int32_t idj = __shfl_sync(0xffffffffu, id, j);
                const double dd = dist_f64_warp(data + int64_t(idj) * dim, qv, dim, metric,
                                                cos ? xnorm[idj] : 1.0, qn, lane);
                if (lane == j) d = dd;
            }
        } else if (need) {
            d = dist_f64_lane(data + int64_t(id) * dim, qv, dim, metric, cos ? xnorm[id] : 1.0, qn);
        }
        if (need) err = fmax(err, fabs(double(approx) - d));
        uint32_t am = __ballot_sync(0xffffffffu, has);
        while (am) {
            const int j = __ffs(am) - 1;
            am &= am - 1;
            const double xd = __shfl_sync(0xffffffffu, d, j);
            const int32_t xi = __shfl_sync(0xffffffffu, id, j);
            if (a == k && !pair_lt(xd, xi, Ad[k - 1], Ai[k - 1])) continue;
            int c = 0;
            for (int r = lane; r < a; r += 32) c += pair_lt(Ad[r], Ai[r], xd, xi);
            const int pos = __reduce_add_sync(0xffffffffu, c);
            for (int top = a - 1; top >= pos; top -= 32) {
                const int r = top - lane;
                double dv = 0;
                int32_t iv = 0;
                if (r >= pos) {
                    dv = Ad[r];
                    iv = Ai[r];
                }
                __syncwarp();
                if (r >= pos) {
                    Ad[r + 1] = dv;
                    Ai[r + 1] = iv;
                }
                __syncwarp();
            }
            if (lane == 0) {
                Ad[pos] = xd;
                Ai[pos] = xi;
            }
            __syncwarp();
            a = min(a + 1, k);
        }
    }
    if (exact_lim > 0.f) {  // results r = q, q + VERIFY_EVERY, ... (mod VERIFY_EVERY) in float64
        bool bad = false;
        const int r0 = q % VERIFY_EVERY;
        if (dim >= COOP_DIM) {
            for (int r = r0; r < a; r += VERIFY_EVERY) {
                const double dd = dist_f64_warp(data + int64_t(Ai[r]) * dim, qv, dim, metric, 1.0, qn, lane);
                bad |= dd != Ad[r];
            }
        } else {
            for (int r = r0 + lane * VERIFY_EVERY; r < a; r += 32 * VERIFY_EVERY)
                bad |= dist_f64_lane(data + int64_t(Ai[r]) * dim, qv, dim, metric, 1.0, qn) != Ad[r];
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(mismatch, 1);
    }
    for (int r = lane; r < k; r += 32) {
        out_ids[int64_t(q) * k + r] = r < a ? int64_t(Ai[r]) : -1;
        out_d[int64_t(q) * k + r] = r < a ? Ad[r] : INFINITY;
    }
    // Non-negative doubles order as their bit patterns: an integer maximum over the warp, then
    // one atomic per query.
    unsigned long long eb = static_cast<unsigned long long>(__double_as_longlong(err));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) eb = max(eb, __shfl_xor_sync(0xffffffffu, eb, o));
    if (lane == 0 && eb) atomicMax(err_max, eb);
}

// Value classes of a float array: *flag gets bit 1 when a value is not an integer with |v| <= 256
// (exact in BF16), bit 2 when one is not an integer in [0, 255] (a byte). Written with explicit
// branches and an integer OR across the warp: a form that combined two boolean warp votes set the
// wrong bits on the GPU (every non-integer and 300 read as bytes), this one was checked against
// those values there.
__global__ void check_small_int(const float *x, int64_t count, int32_t *flag) {
    int f = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += int64_t(gridDim.x) * blockDim.x) {
        const float v = x[i];
        const float r = rintf(v);
        if (r != v || !(fabsf(v) <= 256.f)) f |= 1;
        if (r != v || !(v >= 0.f) || !(v <= 255.f)) f |= 2;
    }
    f = int(__reduce_or_sync(0xffffffffu, uint32_t(f)));
    if (f && (threadIdx.x & 31) == 0) atomicOr(flag, f);
}

// Largest and total of the segment counts (overflow check and the candidate total).
__global__ void count_stats(const int32_t *cnt, int64_t len, unsigned long long *out) {
    unsigned long long mx = 0, sum = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len;
         i += int64_t(gridDim.x) * blockDim.x) {
        const unsigned long long c = static_cast<unsigned long long>(cnt[i]);
        mx = max(mx, c);
        sum += c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, mx);
        atomicAdd(out + 1, sum);
    }
}

// Error bound of the filter arithmetic and the per-query margins (2 e_q).
// Largest of n non-negative doubles: their bit patterns order as unsigned integers.
__global__ void max_norm_kernel(const double *xn, int64_t n, unsigned long long *out) {
    unsigned long long m = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        m = max(m, static_cast<unsigned long long>(__double_as_longlong(xn[i])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void margins_kernel(const double *qnorm, int32_t nq, double xmax, int kp, int terms,
                               int metric, float *margin) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const double qn = metric == HNSW_B200_COSINE ? 1.0 : qnorm[q];
    const double xm = metric == HNSW_B200_COSINE ? 1.0 : xmax;
    const double rep = terms == 1 ? 0.0 : ldexp(1.0, -15);          // dropped lo.lo and rounding
    const double acc = double(kp + 8) * ldexp(1.0, -22);             // FP32 accumulation (2u per add)
    const double e_dot = (rep + acc) * 1.25 * qn * xm;
    double e = e_dot;
    if (metric == HNSW_B200_L2) e = 2.0 * e_dot + ldexp(1.0, -20) * (qn + xm) * (qn + xm);
    else e = e_dot + ldexp(1.0, -22);
    margin[q] = float(2.0 * e * 1.0001);
}

// ============================================================================== host
using hb::fail;

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Tiled map of a row-major operand of kpad elements a row: boxes of one 128-byte swizzle row (BK
// BF16 or BK8 bytes) by box_rows rows.
int make_map(CUtensorMap *map, const void *base, int64_t rows, int kpad, int box_rows, bool u8 = false) {
    auto fn = encode_fn();
    if (!fn) return fail(HNSW_B200_ECUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {cuuint64_t(kpad), cuuint64_t(rows)};
    cuuint64_t strides[1] = {cuuint64_t(kpad) * (u8 ? 1 : 2)};
    cuuint32_t box[2] = {cuuint32_t(u8 ? BK8 : BK), cuuint32_t(box_rows)};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, u8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                    const_cast<void *>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(HNSW_B200_ECUDA, "cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
    return 0;
}

struct Scratch {
    void *p = nullptr;
    size_t bytes = 0;
    ~Scratch() {
        if (p) cudaFree(p);
    }
    int get(size_t b) {
        if (b <= bytes) return 0;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, b) != cudaSuccess) {
            cudaGetLastError();
            return fail(HNSW_B200_ENOMEM, "exact knn scratch allocation failed");
        }
        bytes = b;
        return 0;
    }
};

#define XT(expr)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) return fail(HNSW_B200_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Candidate lists take at most CAND_BYTES of scratch: (query, segment) pairs x cap x 8 bytes.
constexpr int64_t CAND_BYTES = int64_t(4) << 30;
// Pass two keeps about k n / prefix rows per query: tau is the k-th smallest of the prefix's CW-row
// block minima, a loose upper bound of the k-th distance (830 per query measured for k = 100 on the
// 1M x 128 mixture with a prefix of n / 8, against 800 for k n / prefix). Lists are sized for
// EXPECT_FACTOR times that.
#ifndef HB_EXPECT_FACTOR
#define HB_EXPECT_FACTOR 2
#endif
constexpr int64_t EXPECT_FACTOR = HB_EXPECT_FACTOR;
// Byte rows use the integer filter (1) or the BF16 one (0).
#ifndef HB_EXACT_I8
#define HB_EXACT_I8 1
#endif
// Longest byte row of the integer filter: 2 dim 255^2 stays below 2^31.
constexpr int MAX_DIM_I8 = 8192;
// Prefix length. Pass one costs the prefix's rows on the tensor cores; pass two then keeps about
// k n / prefix rows per query, each re-scored in float64 (and a per-element epilogue path on the
// chunks holding them). A float64 re-score of a row costs about PREFIX_BALANCE times a row of
// tensor-core filter work, so the prefix balancing the two is sqrt(PREFIX_BALANCE k n): 122K rows
// for k = 100 over 1M rows (830 candidates per query), 30K over 60K rows.
constexpr double PREFIX_BALANCE = 150.0;


// One attempt at the whole batch with candidate lists of at least cap_min entries. Returns
// HNSW_B200_ERETRY with *cap_needed set when a query's candidates outgrew its list (many rows
// within the margin of the k-th distance, e.g. exact ties); the caller retries with that size.
template <typename T>
int exact_knn_typed(const hnsw_b200_exact_args_t *a, cudaStream_t s, int64_t cap_min,
                    int64_t *cap_needed) {
    const int64_t n = a->n, nq_all = a->nq;
    const int dim = a->dim, k = a->k, metric = a->metric;
    int integer = a->integer_valued;
    // Byte rows (every value an integer in [0, 255], L2 or inner product, int32-safe sums) take the
    // integer tensor-core filter, whose values are the exact distances.
    const bool bytes_ok = HB_EXACT_I8 && metric != HNSW_B200_COSINE && dim <= MAX_DIM_I8;
    bool bytes = false;
    if constexpr (std::is_same_v<T, uint8_t>) {
        integer = 1;
        bytes = bytes_ok;
    } else if (integer != 0) {  // find out on the device, one pass over each array
        static thread_local Scratch flag_buf;
        if (int rc = flag_buf.get(16)) return rc;
        int32_t *flag = static_cast<int32_t *>(flag_buf.p);
        XT(cudaMemsetAsync(flag, 0, 4, s));
        check_small_int<<<1024, 256, 0, s>>>(static_cast<const float *>(a->data), n * dim, flag);
        check_small_int<<<256, 256, 0, s>>>(static_cast<const float *>(a->queries), nq_all * dim, flag);
        XT(cudaGetLastError());
        int32_t hflag = 0;
        XT(cudaMemcpyAsync(&hflag, flag, 4, cudaMemcpyDeviceToHost, s));
        XT(cudaStreamSynchronize(s));
        if (integer < 0) integer = (hflag & 1) ? 0 : 1;
        bytes = bytes_ok && (hflag & 3) == 0;
    }
    const int terms = integer && metric != HNSW_B200_COSINE ? 1 : 3;
    const int seg = (dim + BK - 1) / BK * BK;
    // K of a row: BF16 elements (terms segments), or bytes in 128-byte chunks
    const int kp = bytes ? (dim + BK8 - 1) / BK8 * BK8 : seg * terms;
    const int64_t n_pad = (n + BN - 1) / BN * BN;
    int sms = 148;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    // Split geometry of a pass over `rows` rows for a chunk of nqc queries: the rows are split so
    // that the chunk's query tiles fill the GPU (about four CTAs per SM).
    struct Geo {
        int tps, splits;
    };
    auto geo = [&](int64_t nqc, int64_t rows) {
        const int qt = int((nqc + BM - 1) / BM);
        const int tiles = int((rows + BN - 1) / BN);
        const int want = std::max(1, (4 * sms + qt - 1) / qt);
        Geo g;
        g.tps = std::max(1, (tiles + want - 1) / want);
        g.splits = (tiles + g.tps - 1) / g.tps;
        return g;
    };
    // Pass one keeps the minimum of every (tile, epilogue part) block of a prefix (every row when
    // the prefix has fewer than k such blocks in whole tiles); pass two keeps the rows within tau +
    // margin, about EXPECT_FACTOR k n / prefix of them. Each epilogue thread appends to its own
    // segment of the query's list: in pass one at most one entry per tile (block minima) or CW
    // (rows) per chunk it takes of a tile; pass two's segments are sized for three times their
    // expected share (an overflow re-runs the call with longer segments).
    const int64_t prefix = std::min<int64_t>(
        n, std::max<int64_t>(int64_t(64) * k, int64_t(std::sqrt(PREFIX_BALANCE * double(k) * double(n)))));
    const bool block_min = prefix / BN * EPI_PER_QUARTER >= k;
    const int64_t expect2 = EXPECT_FACTOR * int64_t(k) * ((n + prefix - 1) / prefix) + int64_t(k);
    int64_t QB = std::min<int64_t>(nq_all, 8192);  // queries per chunk
    int64_t cap = 0, slots = 0;                      // entries per segment; (query, segment) pairs
    for (;;) {
        cap = std::min<int64_t>(cap_min, n);
        slots = 0;
        const int64_t last = nq_all % QB ? nq_all % QB : QB;
        for (int64_t nqc : {QB, last}) {
            const Geo g1 = geo(nqc, prefix), g2 = geo(nqc, n);
            const int64_t nseg2 = int64_t(g2.splits) * EPI_PER_QUARTER;
            const int64_t per_tile = (BN / CW + EPI_PER_QUARTER - 1) / EPI_PER_QUARTER;  // chunks
            cap = std::max<int64_t>(cap, per_tile * (block_min ? 1 : CW) * g1.tps);
            cap = std::max<int64_t>(cap, (3 * expect2 + nseg2 - 1) / nseg2 + 32);
            slots = std::max<int64_t>(slots, nqc * std::max(g1.splits, g2.splits) * EPI_PER_QUARTER);
        }
        if (slots * cap * 8 <= CAND_BYTES || QB <= BM) break;
        QB = std::max<int64_t>(BM, QB / 2 / BM * BM);  // longer lists: fewer queries per chunk
    }
    const int64_t q_pad = (QB + BM - 1) / BM * BM;
    static thread_local Scratch buf;
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        size_t o = off;
        off += al256(bytes);
        return o;
    };
    const size_t esz = bytes ? 1 : 2;  // operand element bytes
    const size_t o_xb = carve(size_t(n_pad) * kp * esz);
    const size_t o_qb = carve(size_t(q_pad) * kp * esz);
    const size_t o_xn = carve(size_t(n_pad) * 8);
    const size_t o_qn = carve(size_t(q_pad) * 8);
    const size_t o_xx = carve(size_t(n_pad) * 4);
    const size_t o_qq = carve(size_t(q_pad) * 4);
    const size_t o_mg = carve(size_t(QB) * 4);
    const size_t o_th = carve(size_t(QB) * 4);
    const size_t o_tau = carve(size_t(QB) * 4);
    const size_t o_cnt = carve(size_t(slots) * 4);
    const size_t o_cm = carve(size_t(QB) * 4);
    const size_t o_cv = carve(size_t(slots) * cap * 4);
    const size_t o_ci = carve(size_t(slots) * cap * 4);
    const size_t o_cs = carve(16);
    const size_t o_err = carve(16);
    const size_t o_mx = carve(16);
    const size_t o_fe = carve(16);
    if (int rc = buf.get(off)) return rc;
    char *B = static_cast<char *>(buf.p);
    auto *xb = reinterpret_cast<__nv_bfloat16 *>(B + o_xb);
    auto *qb = reinterpret_cast<__nv_bfloat16 *>(B + o_qb);
    auto *xn = reinterpret_cast<double *>(B + o_xn);
    auto *qn = reinterpret_cast<double *>(B + o_qn);
    auto *xx = reinterpret_cast<float *>(B + o_xx);
    auto *qq = reinterpret_cast<float *>(B + o_qq);
    auto *xb8 = reinterpret_cast<uint8_t *>(B + o_xb);  // byte path: the same buffers as u8 / int32
    auto *qb8 = reinterpret_cast<uint8_t *>(B + o_qb);
    auto *xxi = reinterpret_cast<int32_t *>(B + o_xx);
    auto *qqi = reinterpret_cast<int32_t *>(B + o_qq);
    auto *mg = reinterpret_cast<float *>(B + o_mg);
    auto *th = reinterpret_cast<float *>(B + o_th);
    auto *tau = reinterpret_cast<float *>(B + o_tau);
    auto *cnt = reinterpret_cast<int32_t *>(B + o_cnt);
    auto *cm = reinterpret_cast<int32_t *>(B + o_cm);  // per query: candidates after compaction
    auto *cv = reinterpret_cast<float *>(B + o_cv);
    auto *ci = reinterpret_cast<int32_t *>(B + o_ci);
    auto *err = reinterpret_cast<int32_t *>(B + o_err);
    const T *X = static_cast<const T *>(a->data);
    const int cos = metric == HNSW_B200_COSINE;
    int64_t launches = 0;

    if (bytes)
        prep_rows_u8<T><<<int(std::min<int64_t>(4096, (n_pad + 7) / 8)), 256, 0, s>>>(
            X, n, dim, n_pad, kp, xb8, xxi);
    else
        prep_rows<T><<<int(std::min<int64_t>(4096, (n_pad + 7) / 8)), 256, 0, s>>>(
            X, n, dim, n_pad, kp, terms, 0, cos, xb, xn, xx);
    XT(cudaGetLastError());
    launches++;
    double xmax = 1.0;  // largest data norm (margins): a device reduction, one 8-byte copy
    if (!cos && !bytes) {
        auto *mx = reinterpret_cast<unsigned long long *>(B + o_mx);
        XT(cudaMemsetAsync(mx, 0, 8, s));
        max_norm_kernel<<<int(std::min<int64_t>(1024, (n + 255) / 256)), 256, 0, s>>>(xn, n, mx);
        XT(cudaGetLastError());
        unsigned long long bits = 0;
        XT(cudaMemcpyAsync(&bits, mx, 8, cudaMemcpyDeviceToHost, s));
        XT(cudaStreamSynchronize(s));
        std::memcpy(&xmax, &bits, 8);
        launches++;
    }
    CUtensorMap tmA, tmB;
    if (int rc = make_map(&tmA, B + o_qb, q_pad, kp, BM, bytes)) return rc;
    if (int rc = make_map(&tmB, B + o_xb, n_pad, kp, BN, bytes)) return rc;
    const size_t smem = STAGES * STAGE_BYTES + XSLOTS * BN * 4 + 1024 + BAR_BYTES;
    XT(cudaFuncSetAttribute(knn_filter_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    XT(cudaFuncSetAttribute(knn_filter_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int wpb = 4;
    const size_t rsm = size_t(wpb) * (k + 1) * 12;
    if (rsm > 200 * 1024) return fail(HNSW_B200_EINVAL, "k too large for the rerank kernel");
    XT(cudaFuncSetAttribute(rerank_topk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(rsm)));
    XT(cudaMemsetAsync(err, 0, 16, s));
    auto *ferr = reinterpret_cast<unsigned long long *>(B + o_fe);  // measured filter error (bits)
    XT(cudaMemsetAsync(ferr, 0, 8, s));
    std::vector<float> inf(static_cast<size_t>(QB), INFINITY);
    auto *cstat = reinterpret_cast<unsigned long long *>(B + o_cs);  // largest and total count
    double max_margin = 0.0;
    int64_t total_cand = 0;

    for (int64_t q0 = 0; q0 < nq_all; q0 += QB) {
        const int64_t nq = std::min<int64_t>(QB, nq_all - q0);
        const T *Q = static_cast<const T *>(a->queries) + q0 * dim;
        if (bytes) {  // exact filter values: no margin
            prep_rows_u8<T><<<int(std::min<int64_t>(4096, (q_pad + 7) / 8)), 256, 0, s>>>(
                Q, nq, dim, q_pad, kp, qb8, qqi);
            XT(cudaMemsetAsync(mg, 0, size_t(nq) * 4, s));
        } else {
            prep_rows<T><<<int(std::min<int64_t>(4096, (q_pad + 7) / 8)), 256, 0, s>>>(
                Q, nq, dim, q_pad, kp, terms, 1, cos, qb, qn, qq);
            margins_kernel<<<int((nq + 255) / 256), 256, 0, s>>>(qn, int32_t(nq), xmax, kp, terms, metric, mg);
        }
        XT(cudaGetLastError());
        launches += 2;
        // Query tiles of this chunk only (the last chunk may be short), rows split to fill the GPU.
        const int qt_chunk = int((nq + BM - 1) / BM);
        int nseg = 0;  // segments per query of the last pass run
        auto run_filter = [&](int64_t row_end, bool bmin) -> int {
            const Geo gg = geo(nq, row_end);
            const int tps = gg.tps, splits = gg.splits;
            nseg = splits * EPI_PER_QUARTER;
            FilterParams fp;
            fp.nq = int32_t(nq);
            fp.row_begin = 0;
            fp.row_end = int32_t(row_end);
            fp.kchunks = kp / (bytes ? BK8 : BK);
            fp.tiles_per_split = tps;
            fp.metric = metric;
            fp.qq = qq;
            fp.xx = xx;
            fp.qqi = qqi;
            fp.xxi = xxi;
            fp.thr = th;
            fp.cand_val = cv;
            fp.cand_id = ci;
            fp.cand_cnt = cnt;
            fp.cap = int32_t(cap);
            fp.block_min = bmin ? 1 : 0;
            fp.err = err;
            if (bytes)
                knn_filter_kernel<true><<<dim3(qt_chunk, splits), FILTER_THREADS, smem, s>>>(tmA, tmB, fp);
            else
                knn_filter_kernel<false><<<dim3(qt_chunk, splits), FILTER_THREADS, smem, s>>>(tmA, tmB, fp);
            XT(cudaGetLastError());
            launches++;
            return 0;
        };
        // Pass one: the prefix rows with no threshold give tau (an upper bound of the k-th).
        XT(cudaMemcpyAsync(th, inf.data(), size_t(nq) * 4, cudaMemcpyHostToDevice, s));
        // One candidate per CW-row block suffices while the prefix has at least k blocks.
        if (int rc = run_filter(prefix, block_min)) return rc;
        // tau: the k-th smallest block minimum (a warp per query over its compacted list; a block
        // per query over the segments measured 11% slower on the 60K x 784 set).
        select_kth<<<int((nq + SELECT_WARPS - 1) / SELECT_WARPS), 32 * SELECT_WARPS, 0, s>>>(
            cv, nullptr, cnt, int32_t(cap), int32_t(nseg), int32_t(nq), k, mg, th, tau, cm);
        // Pass two: every row against tau + margin.
        if (int rc = run_filter(n, false)) return rc;
        XT(cudaMemsetAsync(cstat, 0, 16, s));
        count_stats<<<int(std::min<int64_t>(1024, (nq * nseg + 255) / 256)), 256, 0, s>>>(
            cnt, nq * nseg, cstat);
        XT(cudaGetLastError());
        launches++;
        int32_t herr[4];
        unsigned long long hst[2];
        XT(cudaMemcpyAsync(hst, cstat, 16, cudaMemcpyDeviceToHost, s));
        XT(cudaMemcpyAsync(herr, err, 16, cudaMemcpyDeviceToHost, s));
        XT(cudaStreamSynchronize(s));
        if (herr[0]) return fail(HNSW_B200_ECUDA, "exact knn: a bounded wait expired in the filter kernel");
        const int64_t worst = int64_t(hst[0]);
        total_cand += int64_t(hst[1]);
        if (worst > cap) {
            *cap_needed = worst;
            return fail(HNSW_B200_ERETRY, "exact knn: candidate buffer overflow (" + std::to_string(worst) +
                                              " > " + std::to_string(cap) + ")");
        }
        // The k-th smallest candidate is the global k-th approximate distance: final threshold.
        select_kth<<<int((nq + SELECT_WARPS - 1) / SELECT_WARPS), 32 * SELECT_WARPS, 0, s>>>(
            cv, ci, cnt, int32_t(cap), int32_t(nseg), int32_t(nq), k, mg, th, tau, cm);
        rerank_topk<T><<<int((nq + wpb - 1) / wpb), wpb * 32, rsm, s>>>(
            X, Q, dim, int32_t(nq), k, metric, xn, qn, cv, ci, cm, int32_t(cap), int32_t(nseg), th,
            a->out_ids + q0 * k, a->out_dists + q0 * k, ferr, bytes ? EXACT_LIM : 0.f, err + 1);
        XT(cudaGetLastError());
        launches += 3;
        if (a->out_filter_error_bound) {
            // BF16 filter: half the largest margin. Byte rows: the integer distances are exact and
            // only their float copies of 2^24 or more round, by at most half a float ulp of the
            // final threshold (counted here as a margin of a whole ulp).
            std::vector<float> hm(static_cast<size_t>(nq));
            XT(cudaMemcpyAsync(hm.data(), bytes ? th : mg, size_t(nq) * 4, cudaMemcpyDeviceToHost, s));
            XT(cudaStreamSynchronize(s));
            for (float v : hm) {
                // inner product: candidates reach below the threshold, down to -dim 255^2
                if (bytes && metric == HNSW_B200_IP) v = float(dim) * 65025.f;
                if (!bytes) {
                    max_margin = std::max(max_margin, double(v));
                } else if (std::fabs(v) >= EXACT_LIM && std::isfinite(v)) {
                    int e = 0;
                    std::frexp(double(std::fabs(v)), &e);  // |v| in [2^(e-1), 2^e)
                    max_margin = std::max(max_margin, std::ldexp(1.0, e - 24));
                }
            }
        }
    }
    if (bytes) {  // the integer results against their float64 re-scores
        int32_t hm[4];
        XT(cudaMemcpyAsync(hm, err, 16, cudaMemcpyDeviceToHost, s));
        XT(cudaStreamSynchronize(s));
        if (hm[1]) return fail(HNSW_B200_ECUDA, "exact knn: an integer filter distance differs from its float64 re-score");
    }
    if (a->out_filter_error_bound) *a->out_filter_error_bound = max_margin / 2.0;
    if (a->out_filter_max_error) {
        unsigned long long bits = 0;
        XT(cudaMemcpyAsync(&bits, ferr, 8, cudaMemcpyDeviceToHost, s));
        XT(cudaStreamSynchronize(s));
        double e = 0.0;
        std::memcpy(&e, &bits, 8);
        *a->out_filter_max_error = e;
    }
    if (a->out_candidates) *a->out_candidates = total_cand;
    if (a->out_launches) *a->out_launches = launches;
    return 0;
}

}  // namespace hbx

extern "C" int hnsw_b200_exact_knn(const hnsw_b200_exact_args_t *a, void *stream) {
    using namespace hbx;
    if (!a || !a->data || !a->queries || !a->out_ids || !a->out_dists)
        return fail(HNSW_B200_EINVAL, "null argument");
    if (a->n < 1 || a->n > 0x7ffffff0 || a->dim < 1 || a->k < 1 || a->k > a->n || a->nq < 0)
        return fail(HNSW_B200_EINVAL, "need n >= 1, dim >= 1, 1 <= k <= n");
    if (a->metric < 0 || a->metric > 2) return fail(HNSW_B200_EINVAL, "unknown metric");
    if (a->nq == 0) return 0;
    if (a->dtype != HNSW_B200_F32 && a->dtype != HNSW_B200_U8)
        return fail(HNSW_B200_EINVAL, "unsupported dtype");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // A candidate overflow re-runs the batch with lists long enough for the largest count seen
    // (plus a quarter); a list of n entries can never overflow, so this ends.
    int64_t cap_min = 0;
    for (int attempt = 0; attempt < 4; attempt++) {
        int64_t need = 0;
        const int rc = a->dtype == HNSW_B200_F32 ? exact_knn_typed<float>(a, s, cap_min, &need)
                                                 : exact_knn_typed<uint8_t>(a, s, cap_min, &need);
        if (rc != HNSW_B200_ERETRY || need <= 0) return rc;
        cap_min = std::max(cap_min, need + need / 4 + 64);
    }
    return fail(HNSW_B200_ERETRY, "exact knn: candidate lists still overflowed after retries");
}
