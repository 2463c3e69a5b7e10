// Pageable host <-> device copies through a pinned staging ring filled and drained by a pool of
// host threads (HostStager in svdi_internal.cuh).
//
// The reference's FIpipe (archive/FIPkernels.cu:679-911) uploads the caller's pageable Visreal,
// Visimag and Bin arrays and downloads the image with plain cudaMemcpy calls; at 8.4 M samples
// that is 167 MB up and 16.8 MB down per call, and the driver's single-threaded staging of
// pageable memory takes most of the call. Here an upload is cut into 16 MB chunks: the pool copies
// chunk k into a free slot (each thread one 4 KB-aligned slice) while the copy engine moves chunk
// k - 1 from its slot to the device; a slot is reused once the event recorded after its DMA has
// completed. A download runs the same ring the other way.
#include "svdi_internal.cuh"

#include <algorithm>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

namespace svdi {

namespace {
constexpr size_t kSlotBytes = size_t(16) << 20;
constexpr int kSlots = 3;
constexpr size_t kMinStaged = size_t(4) << 20;  // smaller copies: the driver's staging is as fast
constexpr size_t kMinParallel = size_t(1) << 20;
constexpr size_t kSliceAlign = 4096;
constexpr int kMaxThreads = 8;  // default cap; SVDI_HOST_COPY_THREADS overrides it
}  // namespace

struct HostStager::Impl {
    // the pool: thread w (1 .. nthreads - 1) copies slice w of the current job, the calling thread
    // slice 0
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_job, cv_done;
    unsigned long long gen = 0;
    int remaining = 0;
    bool stop = false;
    char* dst = nullptr;
    const char* src = nullptr;
    size_t bytes = 0, slice = 0;
    int nthreads = 1;
    // the ring
    char* ring = nullptr;
    cudaEvent_t ev[kSlots] = {};
    bool used[kSlots] = {};
    int next = 0;

    void copy_slice(int w) const {
        const size_t lo = (size_t)w * slice;
        if (lo >= bytes) return;
        memcpy(dst + lo, src + lo, std::min(slice, bytes - lo));
    }

    void worker(int w) {
        unsigned long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_job.wait(lk, [&] { return stop || gen != seen; });
                if (stop) return;
                seen = gen;
            }
            copy_slice(w);
            std::lock_guard<std::mutex> lk(mu);
            if (--remaining == 0) cv_done.notify_one();
        }
    }

    void copy(void* d, const void* s, size_t n) {
        if (nthreads == 1 || n < kMinParallel) {
            memcpy(d, s, n);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            dst = static_cast<char*>(d);
            src = static_cast<const char*>(s);
            bytes = n;
            slice = ((n + nthreads - 1) / nthreads + kSliceAlign - 1) / kSliceAlign * kSliceAlign;
            remaining = nthreads - 1;
            ++gen;
        }
        cv_job.notify_all();
        copy_slice(0);
        std::unique_lock<std::mutex> lk(mu);
        cv_done.wait(lk, [&] { return remaining == 0; });
    }

    char* slot(int s) const { return ring + (size_t)s * kSlotBytes; }

    // waits until slot s's last DMA has completed
    int acquire(int s) {
        if (used[s]) SVDI_CUDA(cudaEventSynchronize(ev[s]));
        used[s] = false;
        return SVDI_OK;
    }

    int release(int s, cudaStream_t st) {
        SVDI_CUDA(cudaEventRecord(ev[s], st));
        used[s] = true;
        return SVDI_OK;
    }
};

HostStager::~HostStager() {
    if (!impl_) return;
    {
        std::lock_guard<std::mutex> lk(impl_->mu);
        impl_->stop = true;
    }
    impl_->cv_job.notify_all();
    for (auto& t : impl_->workers) t.join();
    for (int s = 0; s < kSlots; ++s) {
        if (impl_->used[s]) cudaEventSynchronize(impl_->ev[s]);
        if (impl_->ev[s]) cudaEventDestroy(impl_->ev[s]);
    }
    if (impl_->ring) cudaFreeHost(impl_->ring);
    delete impl_;
}

bool HostStager::pageable(const void* host) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

int HostStager::threads() const { return impl_ ? impl_->nthreads : 0; }

int HostStager::init() {
    if (impl_) return SVDI_OK;
    Impl* p = new Impl();
    cudaError_t e = cudaMallocHost(&p->ring, kSlots * kSlotBytes);
    for (int s = 0; s < kSlots && e == cudaSuccess; ++s) e = cudaEventCreateWithFlags(&p->ev[s], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        cudaGetLastError();  // not left for the next launch check to find
        for (int s = 0; s < kSlots; ++s)
            if (p->ev[s]) cudaEventDestroy(p->ev[s]);
        if (p->ring) cudaFreeHost(p->ring);
        delete p;
        SVDI_CUDA(e);
    }
    const unsigned hw = std::thread::hardware_concurrency();
    p->nthreads = std::max(1, std::min<int>(kMaxThreads, hw ? (int)hw : 1));
    if (const char* env = std::getenv("SVDI_HOST_COPY_THREADS")) {  // 1 .. 64 copy threads
        const int want = std::atoi(env);
        if (want > 0) p->nthreads = std::min(want, 64);
    }
    try {
        for (int w = 1; w < p->nthreads; ++w) p->workers.emplace_back(&Impl::worker, p, w);
    } catch (const std::exception&) {  // fewer threads than asked for: slices for those that started
        p->nthreads = (int)p->workers.size() + 1;
    }
    impl_ = p;
    return SVDI_OK;
}

bool HostStager::staged(const void* host, size_t bytes) {
    if (bytes < kMinStaged || unavailable_ || !pageable(host)) return false;
    if (init() != SVDI_OK) {
        unavailable_ = true;
        set_error("");
        return false;
    }
    return true;
}

int HostStager::h2d(void* dev, const void* host, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return SVDI_OK;
    if (!staged(host, bytes)) {
        SVDI_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st));
        return SVDI_OK;
    }
    Impl& I = *impl_;
    for (size_t off = 0; off < bytes; off += kSlotBytes) {
        const size_t n = std::min(kSlotBytes, bytes - off);
        const int s = I.next;
        I.next = (s + 1) % kSlots;
        SVDI_TRY(I.acquire(s));
        I.copy(I.slot(s), static_cast<const char*>(host) + off, n);
        SVDI_CUDA(cudaMemcpyAsync(static_cast<char*>(dev) + off, I.slot(s), n, cudaMemcpyHostToDevice, st));
        SVDI_TRY(I.release(s, st));
    }
    return SVDI_OK;
}

int HostStager::d2h(void* host, const void* dev, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return SVDI_OK;
    if (!staged(host, bytes)) {
        SVDI_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st));
        SVDI_CUDA(cudaStreamSynchronize(st));
        return SVDI_OK;
    }
    Impl& I = *impl_;
    const size_t nch = (bytes + kSlotBytes - 1) / kSlotBytes;
    const int base = I.next;
    auto slot_of = [&](size_t c) { return (int)((base + c) % kSlots); };
    auto issue = [&](size_t c) -> int {
        const int s = slot_of(c);
        const size_t off = c * kSlotBytes;
        SVDI_TRY(I.acquire(s));
        SVDI_CUDA(cudaMemcpyAsync(I.slot(s), static_cast<const char*>(dev) + off, std::min(kSlotBytes, bytes - off),
                                  cudaMemcpyDeviceToHost, st));
        return I.release(s, st);
    };
    for (size_t c = 0; c < std::min<size_t>(nch, kSlots); ++c) SVDI_TRY(issue(c));
    for (size_t c = 0; c < nch; ++c) {
        const int s = slot_of(c);
        const size_t off = c * kSlotBytes;
        SVDI_TRY(I.acquire(s));
        I.copy(static_cast<char*>(host) + off, I.slot(s), std::min(kSlotBytes, bytes - off));
        if (c + kSlots < nch) SVDI_TRY(issue(c + kSlots));
    }
    I.next = slot_of(nch);
    return SVDI_OK;
}

}  // namespace svdi
