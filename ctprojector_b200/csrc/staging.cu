// staging.cu -- host-side transfer and scratch machinery of the
// reference-compatible entries (the c* host-array calls and the cupy* device
// calls that get no workspace).
//
// * Scratch pool: one stream-ordered memory pool per device that keeps up to
//   kPoolKeep bytes mapped between calls.  The default pool returns its memory
//   to the driver at every synchronisation, and the synchronous reference
//   entries synchronise after every call, so each call paid for mapping its
//   scratch again (about 2 ms per call at the 16-slice 512x512 batch).  Inside
//   a CUDA graph capture the plain stream-ordered allocator is used.
// * Host staging: pageable host arrays cross the PCIe link through two pinned
//   chunks per device.  Worker threads copy between the pageable array and a
//   chunk while the copy engine drains (uploads) or fills (downloads) the
//   other one, so the link runs at pinned speed.  The pages of a freshly
//   allocated output array are faulted in by the workers while the device
//   is still computing the result (a page fault and clear per 4 KB page
//   would otherwise halve the download rate).  Pinned (registered) host
//   arrays are copied directly.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "ctp_common.cuh"

namespace ctp {

namespace {

constexpr uint64_t kPoolKeep = 1ull << 30;     // bytes the scratch pool keeps mapped when idle
constexpr size_t kChunk = 8u << 20;            // pinned staging chunk
constexpr size_t kPiece = 1u << 20;            // bytes per worker task
constexpr size_t kDirect = 256u << 10;         // smaller transfers go straight through the driver

// ------------------------------------------------------------ scratch pool
std::atomic<unsigned long long> g_scratch_allocs{0};  // successful scratch_alloc calls (all devices)
std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;

int device_pool(int dev, cudaMemPool_t* out) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) {
        *out = it->second;
        return CTP_OK;
    }
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return set_error((int)e, "scratch pool: %s", cudaGetErrorString(e));
    uint64_t keep = kPoolKeep;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return set_error((int)e, "scratch pool threshold: %s", cudaGetErrorString(e));
    g_pools[dev] = pool;
    *out = pool;
    return CTP_OK;
}

// ------------------------------------------------------------ worker threads
// A fixed team of threads that runs the tasks [0, n) of one parallel_for at
// a time; the calling thread takes part.  Created on first use and again in a
// forked child (threads do not survive fork).
class Workers {
   public:
    explicit Workers(int n) {
        for (int i = 0; i < n; ++i) threads_.emplace_back([this] { loop(); });
    }
    ~Workers() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    void parallel_for(int n, const std::function<void(int)>& f) {
        std::lock_guard<std::mutex> run(run_mu_);  // one parallel_for at a time
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &f;
            total_ = n;
            next_.store(0);
            remaining_ = n;
            ++gen_;
        }
        cv_.notify_all();
        work();
        // every task has run and no thread still holds this job
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return remaining_ == 0 && active_ == 0; });
        job_ = nullptr;
    }

   private:
    void work() {
        const std::function<void(int)>* f;
        int total;
        {
            std::lock_guard<std::mutex> lk(mu_);
            f = job_;
            total = total_;
            if (!f) return;
            ++active_;
        }
        int done = 0;
        for (int i = next_.fetch_add(1); i < total; i = next_.fetch_add(1)) {
            (*f)(i);
            ++done;
        }
        std::lock_guard<std::mutex> lk(mu_);
        remaining_ -= done;
        if (--active_ == 0 || remaining_ == 0) done_cv_.notify_all();
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex mu_, run_mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* job_ = nullptr;
    int total_ = 0, remaining_ = 0, active_ = 0;
    std::atomic<int> next_{0};
    uint64_t gen_ = 0;
    bool stop_ = false;
};

std::mutex g_workers_mu;
Workers* g_workers = nullptr;  // never destroyed: process-lifetime threads
pid_t g_workers_pid = 0;

Workers& workers() {
    std::lock_guard<std::mutex> lk(g_workers_mu);
    if (!g_workers || g_workers_pid != getpid()) {
        // a forked child inherits the pointer but not the threads: start anew
        unsigned hw = std::thread::hardware_concurrency();
        int n = (int)std::min(7u, hw > 1 ? hw - 1 : 1u);
        g_workers = new Workers(n);
        g_workers_pid = getpid();
    }
    return *g_workers;
}

void parallel_copy(void* dst, const void* src, size_t bytes) {
    const int pieces = (int)((bytes + kPiece - 1) / kPiece);
    if (pieces <= 1) {
        memcpy(dst, src, bytes);
        return;
    }
    workers().parallel_for(pieces, [&](int i) {
        size_t off = (size_t)i * kPiece, n = std::min(kPiece, bytes - off);
        memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, n);
    });
}

// Fault in (and have the kernel clear) the pages of a host output range,
// one write per 4 KB page, spread over the worker team.  Called while the
// device still computes the result, so the copies into the range later run
// at memory speed instead of paying a page fault per page.  The whole range
// is overwritten by the result afterwards.
void prefault(void* dst, size_t bytes) {
    constexpr size_t kPage = 4096;
    char* base = static_cast<char*>(dst);
    const int pieces = (int)((bytes + 4 * kPiece - 1) / (4 * kPiece));
    workers().parallel_for(pieces, [&](int i) {
        const size_t off = (size_t)i * 4 * kPiece, end = std::min(bytes, off + 4 * kPiece);
        volatile char* p = base;
        p[off] = 0;
        for (size_t a = (off + kPage) & ~(kPage - 1); a < end; a += kPage) p[a] = 0;
    });
}

// ------------------------------------------------------------ pinned chunks
struct Staging {
    std::mutex mu;
    char* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};  // an event has been recorded on the chunk
};

std::mutex g_stage_mu;
std::map<int, std::unique_ptr<Staging>> g_stage;

int staging(Staging** out) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_stage_mu);
    auto& slot = g_stage[dev];
    if (!slot) {
        auto st = std::make_unique<Staging>();
        for (int b = 0; b < 2; ++b) {
            cudaError_t e = cudaHostAlloc((void**)&st->pin[b], kChunk, cudaHostAllocPortable);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->ev[b], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                for (int c = 0; c <= b; ++c) {
                    if (st->pin[c]) cudaFreeHost(st->pin[c]);
                    if (st->ev[c]) cudaEventDestroy(st->ev[c]);
                }
                return set_error((int)e, "host staging buffers: %s", cudaGetErrorString(e));
            }
        }
        slot = std::move(st);
    }
    *out = slot.get();
    return CTP_OK;
}

bool host_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

int cuda_rc(cudaError_t e, const char* what) {
    return e == cudaSuccess ? CTP_OK : set_error((int)e, "%s: %s", what, cudaGetErrorString(e));
}

// The chunk's previous copy (recorded on its event) has completed.
int chunk_free(Staging& st, int b) {
    if (!st.used[b]) return CTP_OK;
    return cuda_rc(cudaEventSynchronize(st.ev[b]), "staging wait");
}

}  // namespace

int scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) cudaGetLastError();
    cudaError_t e;
    if (cs != cudaStreamCaptureStatusNone) {
        e = cudaMallocAsync(p, bytes, s);
    } else {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaMemPool_t pool = nullptr;
        int rc = device_pool(dev, &pool);
        if (rc) return rc;
        e = cudaMallocFromPoolAsync(p, bytes, pool, s);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_error((int)e, "scratch allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    g_scratch_allocs.fetch_add(1, std::memory_order_relaxed);
    return CTP_OK;
}

unsigned long long scratch_allocations() { return g_scratch_allocs.load(std::memory_order_relaxed); }

int staged_upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return CTP_OK;
    if (bytes < kDirect || host_pinned(src))
        return cuda_rc(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "host to device copy");
    Staging* st = nullptr;
    int rc = staging(&st);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(st->mu);
    for (size_t off = 0, k = 0; off < bytes; off += kChunk, ++k) {
        const int b = (int)(k & 1);
        const size_t n = std::min(kChunk, bytes - off);
        if ((rc = chunk_free(*st, b))) return rc;
        parallel_copy(st->pin[b], static_cast<const char*>(src) + off, n);
        if ((rc = cuda_rc(cudaMemcpyAsync(static_cast<char*>(dst) + off, st->pin[b], n, cudaMemcpyHostToDevice, s),
                          "host to device copy")))
            return rc;
        if ((rc = cuda_rc(cudaEventRecord(st->ev[b], s), "staging event"))) return rc;
        st->used[b] = true;
    }
    return CTP_OK;
}

int staged_download(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return CTP_OK;
    if (bytes < kDirect || host_pinned(dst)) {
        int rc = cuda_rc(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "device to host copy");
        return rc ? rc : cuda_rc(cudaStreamSynchronize(s), "device to host copy");
    }
    Staging* st = nullptr;
    int rc = staging(&st);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(st->mu);
    const size_t K = (bytes + kChunk - 1) / kChunk;
    auto issue = [&](size_t k) -> int {
        const int b = (int)(k & 1);
        const size_t off = k * kChunk, n = std::min(kChunk, bytes - off);
        int r = chunk_free(*st, b);
        if (r) return r;
        if ((r = cuda_rc(cudaMemcpyAsync(st->pin[b], static_cast<const char*>(src) + off, n, cudaMemcpyDeviceToHost, s),
                         "device to host copy")))
            return r;
        r = cuda_rc(cudaEventRecord(st->ev[b], s), "staging event");
        st->used[b] = true;
        return r;
    };
    if ((rc = issue(0))) return rc;
    if (K > 1 && (rc = issue(1))) return rc;
    prefault(dst, bytes);  // overlaps the computation still running ahead of the copies
    for (size_t k = 0; k < K; ++k) {
        const int b = (int)(k & 1);
        const size_t off = k * kChunk, n = std::min(kChunk, bytes - off);
        if ((rc = cuda_rc(cudaEventSynchronize(st->ev[b]), "device to host copy"))) return rc;
        parallel_copy(static_cast<char*>(dst) + off, st->pin[b], n);
        if (k + 2 < K && (rc = issue(k + 2))) return rc;
    }
    return CTP_OK;
}

}  // namespace ctp
