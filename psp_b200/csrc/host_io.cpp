#include "host_io.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace psp_b200 {

void ParallelMemcpy(void* dst, const void* src, size_t n) {
    const size_t minPart = size_t(4) << 20;
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t parts = std::max<size_t>(1, std::min<size_t>(std::min<size_t>(hw, 16), n / minPart));
    if (parts == 1) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t step = (n + parts - 1) / parts;
    std::vector<std::thread> pool;
    pool.reserve(parts - 1);
    auto piece = [&](size_t i) {
        const size_t b = i * step, e = std::min(n, b + step);
        if (b < e) std::memcpy(static_cast<char*>(dst) + b, static_cast<const char*>(src) + b, e - b);
    };
    for (size_t i = 1; i < parts; ++i) pool.emplace_back(piece, i);
    piece(0);
    for (std::thread& t : pool) t.join();
}

namespace {

// The pinned ring of one device.
struct PinnedRing {
    std::mutex m;
    unsigned char* pinned = nullptr;
    size_t slotBytes = 0;
    cudaEvent_t done[HostIo::kSlots] = {};
    bool used[HostIo::kSlots] = {};

    // Slots of at least min(kChunk, bytes); the caller holds m.
    void Reserve(size_t bytes) {
        const size_t want = std::min(HostIo::kChunk, bytes);
        if (slotBytes >= want) return;
        for (int i = 0; i < HostIo::kSlots; ++i)
            if (used[i]) CUDA_CHECK(cudaEventSynchronize(done[i]));
        if (pinned) CUDA_CHECK(cudaFreeHost(pinned));
        pinned = nullptr;
        slotBytes = 0;
        // grow to the full chunk once a transfer needs more than a quarter of it
        const size_t slot = want > HostIo::kChunk / 4 ? HostIo::kChunk : want;
        CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&pinned), slot * HostIo::kSlots, cudaHostAllocPortable));
        slotBytes = slot;
        for (int i = 0; i < HostIo::kSlots; ++i) {
            if (!done[i]) CUDA_CHECK(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
            used[i] = false;
        }
    }
};

PinnedRing& RingOfCurrentDevice() {
    static std::mutex gm;
    static std::map<int, std::unique_ptr<PinnedRing>> rings;
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(gm);
    std::unique_ptr<PinnedRing>& r = rings[dev];
    if (!r) r.reset(new PinnedRing);
    return *r;
}

}  // namespace

void* HostIo::Device(size_t bytes) {
    if (dev_.bytes < bytes) {
        dev_.Release();
        dev_.Allocate(bytes);
    }
    return dev_.p;
}

void HostIo::ToDevice(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    PinnedRing& R = RingOfCurrentDevice();
    std::lock_guard<std::mutex> g(R.m);
    R.Reserve(bytes);
    for (size_t off = 0, c = 0; off < bytes; off += R.slotBytes, ++c) {
        const int s = (int)(c % kSlots);
        const size_t n = std::min(R.slotBytes, bytes - off);
        unsigned char* slot = R.pinned + (size_t)s * R.slotBytes;
        if (R.used[s]) CUDA_CHECK(cudaEventSynchronize(R.done[s]));  // the slot's previous DMA has finished
        ParallelMemcpy(slot, static_cast<const char*>(src) + off, n);
        CUDA_CHECK(cudaMemcpyAsync(static_cast<char*>(dst) + off, slot, n, cudaMemcpyHostToDevice, st));
        CUDA_CHECK(cudaEventRecord(R.done[s], st));
        R.used[s] = true;
    }
}

void HostIo::ToHost(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    PinnedRing& R = RingOfCurrentDevice();
    std::lock_guard<std::mutex> g(R.m);
    R.Reserve(bytes);
    const size_t nchunks = (bytes + R.slotBytes - 1) / R.slotBytes;
    auto issue = [&](size_t c) {
        const int s = (int)(c % kSlots);
        const size_t off = c * R.slotBytes, n = std::min(R.slotBytes, bytes - off);
        // the slot's previous user (possibly another handle's stream) is done
        if (R.used[s]) CUDA_CHECK(cudaEventSynchronize(R.done[s]));
        CUDA_CHECK(cudaMemcpyAsync(R.pinned + (size_t)s * R.slotBytes, static_cast<const char*>(src) + off, n,
                                   cudaMemcpyDeviceToHost, st));
        CUDA_CHECK(cudaEventRecord(R.done[s], st));
        R.used[s] = true;
    };
    for (size_t c = 0; c < std::min<size_t>(kSlots, nchunks); ++c) issue(c);
    for (size_t c = 0; c < nchunks; ++c) {
        const int s = (int)(c % kSlots);
        const size_t off = c * R.slotBytes, n = std::min(R.slotBytes, bytes - off);
        CUDA_CHECK(cudaEventSynchronize(R.done[s]));
        ParallelMemcpy(static_cast<char*>(dst) + off, R.pinned + (size_t)s * R.slotBytes, n);
        if (c + kSlots < nchunks) issue(c + kSlots);
    }
}

}  // namespace psp_b200
