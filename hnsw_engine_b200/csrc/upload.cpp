// Upload of a float32 query batch. A small persistent pool of host threads reads the values once
// and gathers what the choice of distance arithmetic needs: every value finite, every value an
// integer, minimum and maximum. The choice is then made on the host, so nothing reads the batch
// back from the GPU before the search launch. For contiguous float32 batches this replaces the host
// validator's NaN/inf pass (the reference's _validation.py:30-35, "contains NaN or infinite
// values") and the float32 cast of metrics.py:49-53, a copy for float32 rows.
//
// The batch reaches the GPU one of two ways. Without a staging buffer, the calling thread issues a
// pageable cudaMemcpyAsync during the read (the driver stages it through its own pinned buffers).
// With a page-locked staging buffer, the pool threads copy the rows into it as they read them,
// with streaming (non-temporal) stores, and one asynchronous DMA follows. Measured on the B200 hosts (16 vCPUs),
// 5 MB: the pageable copy takes 0.30 ms; staging by 4 threads plus the DMA 0.22 ms with streaming
// stores, but 0.86 ms with ordinary ones -- a DMA read of lines still dirty in other cores' caches
// is slow there.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>
#include <emmintrin.h>  // SSE2: baseline on every x86-64 host
#include <unistd.h>

#include "hnsw_b200.h"

namespace hb {
int fail(int code, const std::string &msg);
}

namespace {

// Workers wait on a generation counter; run() hands every worker the same job (worker w runs part
// w - 1 when w <= parts), runs `caller` on the calling thread meanwhile, and returns when all are
// done. One run at a time (run_mutex_). The pool is allocated once and never destroyed (its
// detached threads end with the process, and always find it alive); a forked child builds its
// own. Workers start one at a time; if the system refuses a thread, the pool keeps those it has.
class HostPool {
   public:
    void start(int workers) {
        for (int i = 0; i < workers; ++i) {
            try {
                std::thread t([this, i] { loop(i + 1); });
                t.detach();
            } catch (...) {
                break;
            }
            ++workers_;
        }
    }
    int workers() const { return workers_; }

    void run(int parts, const std::function<void(int)> &fn, const std::function<void()> &caller) {
        std::lock_guard<std::mutex> serial(run_mutex_);
        {
            std::lock_guard<std::mutex> lk(m_);
            job_ = &fn;
            parts_ = parts;
            pending_ = workers_;
            ++gen_;
        }
        wake_.notify_all();
        caller();
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return pending_ == 0; });
    }

   private:
    void loop(int idx) {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            wake_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            const std::function<void(int)> *job = job_;
            const int parts = parts_;
            lk.unlock();
            if (idx <= parts) (*job)(idx - 1);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }

    int workers_ = 0;
    std::mutex run_mutex_, m_;
    std::condition_variable wake_, done_;
    const std::function<void(int)> *job_ = nullptr;
    int parts_ = 0, pending_ = 0;
    uint64_t gen_ = 0;
};

// The process's pool, or nullptr if none could be made (the caller then works alone).
HostPool *pool() noexcept {
    static std::mutex m;
    static HostPool *p = nullptr;
    static pid_t owner = 0;
    std::lock_guard<std::mutex> lk(m);
    if (p == nullptr || owner != getpid()) {
        const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
        HostPool *fresh = new (std::nothrow) HostPool();
        if (fresh == nullptr) return nullptr;
        fresh->start(int(std::min(hw - 1, 16u)));
        p = fresh;
        owner = getpid();
    }
    return p;
}

struct Part {
    bool finite = true, integer = true;
    float lo = FLT_MAX, hi = -FLT_MAX;
};

// Scan values [b, e), four at a time with SSE2 (baseline x86-64, so the library runs on any host
// it is copied to).
//  - finite: |x| <= FLT_MAX; NaN compares unordered and fails it, as +-inf does;
//  - integer: x clamped to [-2^23, 2^23] survives truncation to int32 and back (every float32 of
//    larger magnitude is an integer; the clamp sends NaN to -2^23, an integer);
//  - min / max: MINPS / MAXPS with the running value second, so a NaN input leaves it unchanged.
Part scan(const float *__restrict src, float *__restrict stage, int64_t b, int64_t e) {
    const __m128 absmask = _mm_castsi128_ps(_mm_set1_epi32(0x7fffffff));
    const __m128 big = _mm_set1_ps(FLT_MAX);
    const __m128 c_hi = _mm_set1_ps(8388608.0f), c_lo = _mm_set1_ps(-8388608.0f);
    __m128 lo = _mm_set1_ps(FLT_MAX), hi = _mm_set1_ps(-FLT_MAX);
    __m128i bad = _mm_setzero_si128(), frac = _mm_setzero_si128();
    int64_t i = b;
    // stage + b is 16-byte aligned (parts start at multiples of 16 values; the buffer is
    // page-locked memory, page aligned)
    for (; i + 4 <= e; i += 4) {
        const __m128 x = _mm_loadu_ps(src + i);
        if (stage) _mm_stream_ps(stage + i, x);
        bad = _mm_or_si128(bad, _mm_castps_si128(_mm_cmpnle_ps(_mm_and_ps(x, absmask), big)));
        const __m128 y = _mm_min_ps(_mm_max_ps(x, c_lo), c_hi);
        const __m128 t = _mm_cvtepi32_ps(_mm_cvttps_epi32(y));
        frac = _mm_or_si128(frac, _mm_castps_si128(_mm_cmpneq_ps(t, y)));
        lo = _mm_min_ps(x, lo);
        hi = _mm_max_ps(x, hi);
    }
    alignas(16) float l4[4], h4[4];
    _mm_store_ps(l4, lo);
    _mm_store_ps(h4, hi);
    Part p;
    p.finite = _mm_movemask_epi8(bad) == 0;
    p.integer = _mm_movemask_epi8(frac) == 0;
    for (int j = 0; j < 4; ++j) {
        p.lo = std::min(p.lo, l4[j]);
        p.hi = std::max(p.hi, h4[j]);
    }
    for (; i < e; ++i) {  // the last values, one at a time by the same rules
        const float x = src[i];
        if (stage) stage[i] = x;
        if (!(std::fabs(x) <= FLT_MAX)) {
            p.finite = false;
            continue;
        }
        const float y = std::min(std::max(x, -8388608.0f), 8388608.0f);
        if (float(int32_t(y)) != y) p.integer = false;
        p.lo = std::min(p.lo, x);
        p.hi = std::max(p.hi, x);
    }
    if (stage) _mm_sfence();  // the streaming stores are visible before the DMA is issued
    return p;
}

}  // namespace

extern "C" int hnsw_b200_upload_queries(const float *src, float *dst, int64_t count,
                                        int32_t threads, hnsw_b200_value_stats_t *out,
                                        float *staging, void *stream) {
    if (count < 0 || out == nullptr || (count > 0 && src == nullptr))
        return hb::fail(HNSW_B200_EINVAL, "upload_queries: bad argument");
    if (staging != nullptr && (reinterpret_cast<uintptr_t>(staging) & 15u) != 0)
        return hb::fail(HNSW_B200_EINVAL, "upload_queries: staging must be 16-byte aligned");
    float *stage = dst != nullptr ? staging : nullptr;
    cudaError_t copy_err = cudaSuccess;
    const std::function<void()> copy = [&] {  // pageable copy, concurrent with the scan
        if (dst != nullptr && stage == nullptr && count > 0)
            copy_err = cudaMemcpyAsync(dst, src, size_t(count) * sizeof(float),
                                       cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream));
    };
    const std::function<void()> nothing = [] {};
    // at least 64K values (256 KB) per part: below that a wake-up costs more than the scan
    constexpr int64_t MIN_PART = 65536;
    int parts = int(std::min<int64_t>(std::max(1, threads), (count + MIN_PART - 1) / MIN_PART));
    HostPool *hp = parts > 1 ? pool() : nullptr;
    if (hp == nullptr || hp->workers() < 2) parts = 1;
    std::vector<Part> res;
    if (parts <= 1) {
        copy();
        res.push_back(scan(src, stage, 0, count));
    } else {
        parts = std::min(parts, hp->workers());
        res.resize(size_t(parts));
        const int64_t per = ((count + parts - 1) / parts + 15) / 16 * 16;  // aligned part starts
        const std::function<void(int)> job = [&](int i) {
            const int64_t b = std::min(count, int64_t(i) * per);
            res[size_t(i)] = scan(src, stage, b, std::min(count, b + per));
        };
        hp->run(parts, job, stage ? nothing : copy);
    }
    if (stage != nullptr && count > 0)  // one asynchronous DMA of the staged rows
        copy_err = cudaMemcpyAsync(dst, stage, size_t(count) * sizeof(float),
                                   cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream));
    if (copy_err != cudaSuccess)
        return hb::fail(HNSW_B200_ECUDA, std::string("upload_queries: ") + cudaGetErrorString(copy_err));
    Part all;
    for (const Part &r : res) {
        all.finite = all.finite && r.finite;
        all.integer = all.integer && r.integer;
        all.lo = std::min(all.lo, r.lo);
        all.hi = std::max(all.hi, r.hi);
    }
    out->finite = all.finite ? 1 : 0;
    out->integer = all.integer ? 1 : 0;
    out->min = count ? double(all.lo) : 0.0;
    out->max = count ? double(all.hi) : 0.0;
    return HNSW_B200_OK;
}
