#include "host_io.hpp"

#include <algorithm>
#include <cstring>
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

HostIo::~HostIo() {
    for (int i = 0; i < kSlots; ++i)
        if (done_[i]) cudaEventDestroy(done_[i]);
    if (pinned_) cudaFreeHost(pinned_);
}

void* HostIo::Device(size_t bytes) {
    if (dev_.bytes < bytes) {
        dev_.Release();
        dev_.Allocate(bytes);
    }
    return dev_.p;
}

void HostIo::Reserve(size_t bytes) {
    const size_t want = std::min(kChunk, bytes);
    if (slotBytes_ >= want) return;
    for (int i = 0; i < kSlots; ++i)
        if (used_[i]) CUDA_CHECK(cudaEventSynchronize(done_[i]));
    if (pinned_) CUDA_CHECK(cudaFreeHost(pinned_));
    pinned_ = nullptr;
    CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&pinned_), want * kSlots, cudaHostAllocDefault));
    slotBytes_ = want;
    for (int i = 0; i < kSlots; ++i) {
        if (!done_[i]) CUDA_CHECK(cudaEventCreateWithFlags(&done_[i], cudaEventDisableTiming));
        used_[i] = false;
    }
}

void HostIo::ToDevice(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    Reserve(bytes);
    for (size_t off = 0, c = 0; off < bytes; off += slotBytes_, ++c) {
        const int s = (int)(c % kSlots);
        const size_t n = std::min(slotBytes_, bytes - off);
        unsigned char* slot = pinned_ + (size_t)s * slotBytes_;
        if (used_[s]) CUDA_CHECK(cudaEventSynchronize(done_[s]));  // the slot's previous DMA has finished
        ParallelMemcpy(slot, static_cast<const char*>(src) + off, n);
        CUDA_CHECK(cudaMemcpyAsync(static_cast<char*>(dst) + off, slot, n, cudaMemcpyHostToDevice, st));
        CUDA_CHECK(cudaEventRecord(done_[s], st));
        used_[s] = true;
    }
}

void HostIo::ToHost(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    Reserve(bytes);
    const size_t nchunks = (bytes + slotBytes_ - 1) / slotBytes_;
    auto issue = [&](size_t c) {
        const int s = (int)(c % kSlots);
        const size_t off = c * slotBytes_, n = std::min(slotBytes_, bytes - off);
        CUDA_CHECK(cudaMemcpyAsync(pinned_ + (size_t)s * slotBytes_, static_cast<const char*>(src) + off, n,
                                   cudaMemcpyDeviceToHost, st));
        CUDA_CHECK(cudaEventRecord(done_[s], st));
        used_[s] = true;
    };
    for (size_t c = 0; c < std::min<size_t>(kSlots, nchunks); ++c) issue(c);
    for (size_t c = 0; c < nchunks; ++c) {
        const int s = (int)(c % kSlots);
        const size_t off = c * slotBytes_, n = std::min(slotBytes_, bytes - off);
        CUDA_CHECK(cudaEventSynchronize(done_[s]));
        ParallelMemcpy(static_cast<char*>(dst) + off, pinned_ + (size_t)s * slotBytes_, n);
        if (c + kSlots < nchunks) issue(c + kSlots);
    }
}

}  // namespace psp_b200
