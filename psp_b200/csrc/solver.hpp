// DistHelmholtz on one B200: owns the device state of one Helmholtz problem
// (PSP include/psp/dist_helmholtz.hpp:21-287).
#pragma once
#include <complex>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "analysis.hpp"
#include "kernels.cuh"
#include "profiler.hpp"

namespace psp_b200 {

// Device allocation owned by one object.
struct DeviceBuffer {
    void* p = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { Release(); }
    void Allocate(size_t n);
    void Release();
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// Host staging area whose arrays are uploaded in one copy; device pointers
// are resolved after Upload().
struct TaskArena {
    std::vector<unsigned char> host;
    DeviceBuffer dev;
    template <typename T>
    size_t Push(const std::vector<T>& v) {
        const size_t off = (host.size() + 255) & ~size_t(255);
        host.resize(off + v.size() * sizeof(T));
        if (!v.empty()) std::memcpy(host.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
    void Upload(cudaStream_t st);
    template <typename T>
    T* At(size_t off) const { return reinterpret_cast<T*>(static_cast<unsigned char*>(dev.p) + off); }
};

struct SolveStats {
    int iterations = 0;
    int converged = 0;
    int luckyBreakdown = 0;
    double finalMaxRelResid = 0;
    double seconds = 0;
    double precondSeconds = 0;
    double matvecSeconds = 0;
    double arnoldiSeconds = 0;
    int numPreconditions = 0;
    std::vector<double> history;
};

template <typename R>
class FactorStore;

// GMRES block width for k right-hand sides when availBytes of device memory
// are left and one right-hand side's workspace takes perRhsBytes: the
// widest that fits (at most cap when cap > 0), made equal across blocks and,
// from 16 up, a multiple of 16 when that still fits.  Throws out-of-memory
// with both sizes in the message when not even one fits.
int ChooseBlockWidth(int k, double availBytes, double perRhsBytes, int cap);

// Makes `p` the profiler of launches issued by this thread while in scope.
struct ProfilerBinding {
    Profiler* prev;
    explicit ProfilerBinding(Profiler* p) : prev(CurrentProfiler()) { CurrentProfiler() = p; }
    ~ProfilerBinding() { CurrentProfiler() = prev; }
};

class Helmholtz {
public:
    Helmholtz(const DiscParams& d, double damping, int planesPerPanel, int cutoff, int device);
    ~Helmholtz();

    // Initialize(velocity) (initialize_finalize.hpp:12-377): velocity is a
    // natural-order nx*ny*nz array on the host or (devicePtr) on the device.
    // precision 0: complex-double fronts; 1: complex-single fronts.
    void Initialize(const double* velocity, bool devicePtr, int panelScheme, int precision);
    void Finalize();
    bool Initialized() const { return initialized_; }

    // Solve (solve.hpp:12-56) on a device natural-order [N][k] complex grid, in place.
    // When the GMRES workspace of all k right-hand sides (about N k (m+5)
    // complex doubles) does not fit in device memory, or the environment
    // caps the width (PSP_B200_MAX_RHS_BLOCK), the right-hand sides are
    // solved in blocks one after another: every block converges on its own
    // (the GMRES of one right-hand side never depends on the others), the
    // stats report the largest step count and residual, viewIterates files
    // carry the block's first column (<basename>_rhs<c>-<it>), and Ritz
    // values of right-hand sides whose first cycle was shorter than the
    // longest are padded with NaN.
    void SolveDevice(z64* B, int k, int m, double relTol, SolveStats* stats);
    // B := A B and B := M^{-1} B on device grids (Multiply / Precondition).
    void MultiplyDevice(z64* B, int k);
    void PreconditionDevice(z64* B, int k);
    void SolvePanelDevice(z64* B, int k, int panel);
    // grad (+)= velocity gradient from forward fields U and adjoint fields Z
    // (device natural-order [N][k] grids; grad is a device array of N reals).
    void GradientDevice(const z64* U, const z64* Z, int k, double* grad, bool accumulate);

    const Analysis& analysis() const { return an_; }
    int64_t NumUnknowns() const { return (int64_t)an_.disc.nx * an_.disc.ny * an_.disc.nz; }
    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }
    int precision() const { return precision_; }
    double setupSeconds() const { return setupSeconds_; }
    int64_t factorBytes() const;
    void SetMaxIterations(int n) { maxIterations_ = n; }
    // viewIterates (solve.hpp:579-585): a non-empty basename makes every
    // GMRES inner step that does not converge write the iterate with
    // WriteVolume as <basename>-<it>.
    void SetViewIterates(const std::string& basename) { viewIterates_ = basename; }
    // PRINT_RITZ_VALUES (solve.hpp:257-261, 391-395, 422-426, 589-608) at
    // run time: 0 off, 1 record the Ritz values of the first restart cycle
    // of each Solve, 2 record and print them as the reference does.
    void SetRitzValues(int mode) { ritzMode_ = mode; }
    // Ritz values of the last Solve that recorded them: ritzCount() per
    // right-hand side, right-hand side r at [r * ritzCount() + s].
    const std::vector<std::complex<double>>& ritzValues() const { return ritz_; }
    int ritzCount() const { return ritzCount_; }
    int ritzNumRhs() const { return ritzK_; }
    Profiler& profiler() { return prof_; }
    // Sweep algorithmic flops/bytes for k right-hand sides (0 before Initialize).
    double SweepFlops(int k) const;
    double SweepBytes(int k) const;
    // Panels whose factors stay resident in device memory; the others are
    // re-factored into a per-class slot whenever a sweep reaches them.
    int ResidentPanels() const;
    // Panel factorizations run by sweeps since Initialize (recomputed panels).
    int64_t Refactorizations() const;

    // z-panel pipeline ranks: only panels [p0, p1) are factored by this
    // handle (set before its first Initialize); panel solves of the others
    // are refused.
    void SetPanelRange(int p0, int p1);
    // Panel p's solve on a slab of the grid whose first stored plane is z =
    // zBase (inMode / outAccumulate as in the sweep: 0 B_i; 1 B_i - A_{i,i-1}
    // B_{i-1}, reading the plane below the panel; 2 -A_{i,i+1} B_{i+1}
    // only, reading the plane above; outAccumulate adds the result).
    void SolvePanelSlab(z64* B, int k, int panel, int inMode, int outAccumulate, int zBase);
    // Y := A X (or Y := Bv - A X when Bv is given) on planes [zFirst, zFirst +
    // zCount) of slabs X, Y (and Bv) whose first stored plane is zSlab; X
    // must hold the planes next to that range that exist in the grid.
    void MultiplySlab(const z64* X, z64* Y, const z64* Bv, int k, int zFirst, int zCount, int zSlab);

    // Right-hand sides per GMRES block a Solve of k sides with restart m
    // would use now (k when they all fit).
    int SolveBlockWidth(int k, int m) {
        if (!initialized_) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
        if (k < 1 || m < 1) throw PspError(kLogicError, "need k >= 1 and m >= 1");
        return GmresBlockWidth(k, m);
    }

    // Device scratch shared by the factorization transients (Initialize)
    // and the GMRES workspace (Solve), which are never live at the same
    // time.  Grows to `bytes` (its contents and earlier pointers into it
    // are lost when it does) and returns its base.
    void* Scratch(size_t bytes);
    size_t ScratchBytes() const { return pool_.bytes; }

    // Device tables shared with the factor stores.
    StencilParams sp_{};
    AssemblyParams ap_{};
    DeviceBuffer dS1_, dS2_, dS3_, dS3a_;   // values and reciprocals back to back
    DeviceBuffer dVel_;
    DeviceBuffer dNdToNat_[3], dNbrRows_[3], dRel_[3], dLower_[3];
    std::vector<int> s3aOff_;                // per panel
    Analysis an_;
    double damping_;
    int device_;
    int panelBegin_ = 0, panelEnd_ = 1 << 30;  // panel range of a pipeline rank
    cudaStream_t stream_ = nullptr;

private:
    void BuildTables();
    void Precondition(z64* B, int k, bool useGraph);
    // Carves the GMRES workspace for k right-hand sides and restart m (and,
    // for blocked solves, a k-wide copy of a block's columns) from Scratch.
    void EnsureWorkspace(int k, int m, bool withCols);
    void CheckSweepStatus();
    // GMRES over all k columns of B at once (the reference's form).
    void SolveBlock(z64* B, int k, int m, double relTol, SolveStats* stats);
    // Right-hand sides per GMRES block for k sides and restart m: the
    // widest that fits in device memory (or the environment's cap), made
    // equal across blocks and, from 16 up, a multiple of 16 when that still
    // fits.  Throws out-of-memory when not even one right-hand side fits.
    int GmresBlockWidth(int k, int m);
    // Device bytes one right-hand side of a GMRES block needs with restart m.
    double GmresBytesPerRhs(int m) const;

    Profiler prof_;
    bool initialized_ = false;
    int precision_ = 0;
    int maxIterations_ = 0;
    std::string viewIterates_;
    int ritzMode_ = 0, ritzCount_ = 0, ritzK_ = 0, ritzRhsOffset_ = 0;
    std::vector<std::complex<double>> ritz_;
    double setupSeconds_ = 0;
    std::unique_ptr<FactorStore<double>> f64_;
    std::unique_ptr<FactorStore<float>> f32_;
    DeviceBuffer pool_;
    // GMRES workspace, carved from pool_ by EnsureWorkspace
    z64 *wsX_ = nullptr, *wsX0_ = nullptr, *wsW_ = nullptr, *wsB_ = nullptr, *wsV_ = nullptr;
    z64 *wsCols_ = nullptr, *wsY_ = nullptr;
    void* wsPartial_ = nullptr;
    void* wsScal_ = nullptr;
};

}  // namespace psp_b200
