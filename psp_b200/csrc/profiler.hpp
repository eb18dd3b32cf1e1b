// Optional per-category kernel timing with CUDA events on the launching
// stream, plus the algorithmic flops and bytes of each launch (computed on the
// host from the task lists).  Off unless a handle enables it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace psp_b200 {

enum ProfileCategory {
    kProfFactorGemm = 0,   // square batched GEMM tiles of the factorization
    kProfSolveGemm,        // skinny batched GEMM tiles of the panel solves
    kProfLdlDiag,
    kProfLdlTrsm,
    kProfAssemble,
    kProfExtendAdd,
    kProfGatherScatter,    // panel-solve gathers and scatters
    kProfStencil,          // global operator apply
    kProfVector,           // GMRES vector kernels
    kProfSweep,            // one whole preconditioner application
    kProfNumCategories
};

struct ProfileTotals {
    int64_t launches = 0;
    double ms = 0;
    double flops = 0;
    double bytes = 0;
};

class Profiler {
public:
    bool enabled = false;
    void Begin(cudaStream_t st);
    void End(cudaStream_t st, int category, double flops, double bytes);
    void Flush();   // resolves recorded events; the stream must be idle
    void Reset();
    ProfileTotals totals[kProfNumCategories];
    ~Profiler();

private:
    struct Rec {
        cudaEvent_t a, b;
        int cat;
        double flops, bytes;
    };
    std::vector<Rec> pending_;
    std::vector<cudaEvent_t> pool_;
    cudaEvent_t open_ = nullptr;
    cudaEvent_t Get();
};

// The profiler of the handle currently issuing work on this thread (null
// when profiling is off).
Profiler*& CurrentProfiler();

struct ProfScope {
    Profiler* p;
    cudaStream_t st;
    int cat;
    double flops, bytes;
    ProfScope(cudaStream_t s, int c, double f = 0, double b = 0) : p(CurrentProfiler()), st(s), cat(c), flops(f), bytes(b) {
        if (p && p->enabled) p->Begin(st);
    }
    ~ProfScope() {
        if (p && p->enabled) p->End(st, cat, flops, bytes);
    }
};

}  // namespace psp_b200
