#include "common.cuh"
#include "profiler.hpp"

namespace psp_b200 {

Profiler*& CurrentProfiler() {
    static thread_local Profiler* p = nullptr;
    return p;
}

cudaEvent_t Profiler::Get() {
    if (!pool_.empty()) {
        cudaEvent_t e = pool_.back();
        pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    CUDA_CHECK(cudaEventCreate(&e));
    return e;
}

void Profiler::Begin(cudaStream_t st) {
    open_ = Get();
    CUDA_CHECK(cudaEventRecord(open_, st));
}

void Profiler::End(cudaStream_t st, int category, double flops, double bytes) {
    if (!open_) return;
    cudaEvent_t b = Get();
    CUDA_CHECK(cudaEventRecord(b, st));
    pending_.push_back(Rec{open_, b, category, flops, bytes});
    open_ = nullptr;
}

void Profiler::Flush() {
    for (const Rec& r : pending_) {
        float ms = 0;
        CUDA_CHECK(cudaEventSynchronize(r.b));
        CUDA_CHECK(cudaEventElapsedTime(&ms, r.a, r.b));
        ProfileTotals& t = totals[r.cat];
        t.launches += 1;
        t.ms += ms;
        t.flops += r.flops;
        t.bytes += r.bytes;
        pool_.push_back(r.a);
        pool_.push_back(r.b);
    }
    pending_.clear();
}

void Profiler::Reset() {
    Flush();
    for (auto& t : totals) t = ProfileTotals();
}

Profiler::~Profiler() {
    for (const Rec& r : pending_) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
}

}  // namespace psp_b200
