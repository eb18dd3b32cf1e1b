// Host <-> device transfers of caller-owned grids for the C ABI's host-buffer
// entry points (psp_cu_solve, psp_cu_initialize, ...).  The caller's memory
// is ordinary pageable memory; a ring of pinned chunks carries it: host
// threads copy one chunk into pinned memory while the previous chunks are in
// flight over DMA, so a transfer runs near the copy engines' rate instead of
// the driver's pageable-copy rate.  The ring is one per device and process,
// shared by every handle on that device (transfers take turns) and kept
// until the process exits (at most kSlots x kChunk bytes of pinned memory);
// the device scratch the grid lands in is per handle and kept between calls.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "solver.hpp"

namespace psp_b200 {

class HostIo {
public:
    HostIo() = default;
    HostIo(const HostIo&) = delete;
    HostIo& operator=(const HostIo&) = delete;

    // Device scratch of at least `bytes` on the current device, kept until a
    // larger one is needed.
    void* Device(size_t bytes);
    // dst (device) := src (host) on stream st (of the current device).
    // Returns once src may be reused; the copies are ordered before later
    // work on st.
    void ToDevice(void* dst, const void* src, size_t bytes, cudaStream_t st);
    // dst (host) := src (device) after the work queued on st; returns when
    // dst holds the data.
    void ToHost(void* dst, const void* src, size_t bytes, cudaStream_t st);

    static constexpr int kSlots = 3;
    static constexpr size_t kChunk = size_t(64) << 20;

private:
    DeviceBuffer dev_;
};

// Copies n bytes with up to the host's hardware threads (at least 4 MB each).
void ParallelMemcpy(void* dst, const void* src, size_t n);

}  // namespace psp_b200
