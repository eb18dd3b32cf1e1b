// Host orchestration of the B200 sweeping-preconditioned Helmholtz solve:
// table upload, depth-batched multifrontal factorization of every panel,
// the sweep (Precondition, solve.hpp:681-734) and multi-RHS GMRES(m)
// (InternalSolveWithGMRES, solve.hpp:241-611).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "solver.hpp"

#include "grid_io.hpp"
#include "ritz.hpp"

namespace psp_b200 {

void DeviceBuffer::Allocate(size_t n) {
    Release();
    if (n == 0) n = 256;
    CUDA_CHECK(cudaMalloc(&p, n));
    bytes = n;
}

void DeviceBuffer::Release() {
    if (p) {
        cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
}

void TaskArena::Upload(cudaStream_t st) {
    if (host.empty()) host.resize(256);
    if (dev.bytes < host.size()) dev.Allocate(host.size());
    CUDA_CHECK(cudaMemcpyAsync(dev.p, host.data(), host.size(), cudaMemcpyHostToDevice, st));
    CUDA_CHECK(cudaStreamSynchronize(st));
}

namespace {

typedef std::complex<double> Cd;

// Sweep variants (kernel and K-chunk per depth) chosen by timing, shared by
// every handle of the process with the same front structure, block width
// and device: equal problems then run the same kernels (a re-initialized handle and a fresh
// one give identical results) and a batch of equal problems is timed once.
std::mutex gRouteMutex, gTuneMutex;
std::map<std::string, std::vector<int>> gRoutes;

// Imaginary stretch of a PML point at distance `delta` from the inner edge
// (the common body of s1Inv/s2Inv/s3Inv/s3InvArtificial,
// initialize_finalize.hpp:415-525).
Cd PmlPoint(double delta, int b, double sigma, double h, double omega) {
    const double eta = b * h;
    return Cd(1.0, (sigma / eta) * (delta / b) * (delta / b) * (2 * M_PI / omega));
}

// Value of a 1-D stretch at grid index i (low face active for i < b-1 + lowShift).
Cd Stretch(int i, int n, int b, double sigma, double h, double omega, bool lowPML, bool highPML, int lowEdge) {
    if (lowPML && i < lowEdge + b - 1) return PmlPoint((lowEdge + b - 1) - i, b, sigma, h, omega);
    if (highPML && i > n - b) return PmlPoint(i - (n - b), b, sigma, h, omega);
    return Cd(1.0, 0.0);
}

void PushTable(std::vector<z64>& vals, std::vector<z64>& invs, const std::vector<Cd>& t) {
    for (const Cd& c : t) {
        vals.push_back(mk(c.real(), c.imag()));
        const Cd inv = 1.0 / c;
        invs.push_back(mk(inv.real(), inv.imag()));
    }
}

template <typename T>
void UploadVector(DeviceBuffer& buf, const std::vector<T>& v, cudaStream_t st) {
    buf.Allocate(std::max<size_t>(v.size() * sizeof(T), 256));
    if (!v.empty()) CUDA_CHECK(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    CUDA_CHECK(cudaStreamSynchronize(st));
}

// Sum over r < M of the nonzero products in row r of a triangular operand.
double TriRowSum(int64_t M, int64_t K, int tri) {
    if (tri == 1) {  // k <= r
        if (M <= K) return (double)M * (M + 1) / 2;
        return (double)K * (K + 1) / 2 + (double)(M - K) * K;
    }
    if (tri == 2) {  // k >= r
        const int64_t m = std::min(M, K);
        return (double)m * K - (double)m * (m - 1) / 2;
    }
    return (double)M * K;
}

// Algorithmic real flops (8 per complex multiply-add, structural zeros
// skipped) and algorithmic bytes (nonzero operand elements read once, output
// written once and read once when accumulated) of one batched-GEMM op.
template <typename R>
void OpCost(const GemmOp<R>& op, double& flops, double& bytes) {
    double macs, aElems, bElems = (double)op.K * op.N, cElems;
    if (op.lowerC) {
        cElems = (double)op.N * op.M - (double)op.N * (op.N - 1) / 2;
        macs = cElems * op.K;
        aElems = (double)op.M * op.K;
    } else if (op.triA) {
        aElems = TriRowSum(op.M, op.K, op.triA);
        macs = aElems * op.N;
        cElems = (double)op.M * op.N;
    } else if (op.triB) {
        bElems = TriRowSum(op.N, op.K, op.triB == 1 ? 2 : 1);
        macs = bElems * op.M;
        aElems = (double)op.M * op.K;
        cElems = (double)op.M * op.N;
    } else {
        macs = (double)op.M * op.N * op.K;
        aElems = (double)op.M * op.K;
        cElems = (double)op.M * op.N;
    }
    const bool acc = op.beta_re != R(0) || op.beta_im != R(0);
    flops += 8.0 * macs;
    bytes += sizeof(cpx<R>) * (aElems + bElems + cElems * (acc ? 2 : 1));
}

template <typename R>
GemmOp<R> MakeOp(const cpx<R>* A, int64_t lda, int transA, const cpx<R>* B, int64_t ldb, int transB, cpx<R>* C,
                 int64_t ldc, int M, int N, int K, R alpha, R beta) {
    GemmOp<R> op;
    std::memset(&op, 0, sizeof(op));
    op.A = A; op.lda = lda; op.transA = transA;
    op.B = B; op.ldb = ldb; op.transB = transB;
    op.C = C; op.ldc = ldc;
    op.M = M; op.N = N; op.K = K;
    op.alpha_re = alpha; op.beta_re = beta;
    return op;
}

}  // namespace

// =====================================================================
// Factor store: persistent G (selectively inverted factors) and D per
// panel, the factorization schedule and the panel solves.
// =====================================================================

template <typename R>
class FactorStore {
public:
    explicit FactorStore(Helmholtz& h) : h_(h), an_(h.an_) {
        PrepareSweepKernels<R>();
        // Complex-single factors use the tensor-core sweep unless the
        // environment asks for the CUDA-core kernels (for comparisons).
        const char* env = std::getenv("PSP_B200_SWEEP_CUDA_CORES");
        tc_ = std::is_same<R, float>::value && !(env && env[0] == '1');
        if (tc_) PrepareSweepTcKernels();
        // Likewise the factorization GEMMs of complex-single fronts.
        const char* fenv = std::getenv("PSP_B200_FACTOR_CUDA_CORES");
        factorTc_ = std::is_same<R, float>::value && !(fenv && fenv[0] == '1');
        if (factorTc_) PrepareFactorTcKernels();
    }
    ~FactorStore() {
        for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
    }
    void Factor();
    // Makes panel p's factors available: a recomputed panel is factored
    // into its class's slot unless the slot holds it already.
    void EnsurePanel(int p);
    // Panel p's solve on grid B (rows of ldk complex entries per point);
    // B's first stored plane is z = zBase (a slab of the global grid).
    void SolvePanel(z64* B, int ldk, int k, int p, int inMode, int outAcc, int zBase = 0);
    // One sweep (Precondition); replayed from a captured CUDA graph when
    // `useGraph` and profiling is off.
    void Sweep(z64* B, int ldk, int k, bool useGraph);
    int64_t Bytes() const {
        int64_t b = (int64_t)(G_.bytes + D_.bytes);
        for (int c = 0; c < 3; ++c) b += (int64_t)(slotG_[c].bytes + slotD_[c].bytes);
        return b;
    }
    int ResidentPanels() const {
        int n = 0;
        for (char r : resident_) n += r;
        return n;
    }
    int64_t Refactorizations() const { return refactors_; }
    // Device bytes of the solve plan per right-hand side (work vectors).
    double PlanBytesPerRhs() const;
    bool HasPlan(int k) const {
        for (const auto& pl : plans_)
            if (pl->k == k) return true;
        return false;
    }
    // Frees the solve plans (and the sweep graphs that use them) of every
    // block width but k.
    void DropPlansExcept(int k);
    // Device status word: bit 1 zero/non-finite pivot, bit 2 a tensor-core
    // pipeline wait timed out.  Synchronizes the stream.
    int ReadStatus() {
        int st = 0;
        CUDA_CHECK(cudaMemcpyAsync(&st, status_.p, sizeof(int), cudaMemcpyDeviceToHost, h_.stream_));
        CUDA_CHECK(cudaStreamSynchronize(h_.stream_));
        return st;
    }
    double SweepFlops(int k) const;
    double SweepBytes(int k) const;

private:
    struct Step {
        enum Kind { kMemset, kAssemble, kExtend, kDiag, kTrsm, kGemm } kind;
        size_t a = 0, b = 0, c = 0;
        int n = 0, nTc = 0, J = 0;  // n CUDA-core tiles at b, nTc tensor-core tiles at c
        size_t bytes = 0;
        double flops = 0, abytes = 0;
    };
    struct SweepGraph {
        z64* B;
        int ldk, k;
        cudaGraphExec_t exec;
    };
    std::vector<SweepGraph> graphs_;
    void SweepEager(z64* B, int ldk, int k);
    // The factorization of one group of panels as recorded launches: its
    // uploaded task lists and steps, with the transient buffers at a fixed
    // place (the handle's scratch for the resident panels, the recompute
    // arena for a recomputed panel).  Programs are kept, so a later
    // Initialize of the same handle (same structure, new velocity) only
    // replays them while the scratch has not moved.
    struct FactorProgram {
        unsigned char* arena = nullptr;
        size_t arenaBytes = 0;
        TaskArena tasks;
        std::vector<Step> steps;
        size_t frontsOff = 0;
    };
    std::vector<std::unique_ptr<FactorProgram>> program_;
    // Transient bytes of the factorization of `panels` at its busiest depth.
    int64_t TransientBytes(const std::vector<int>& panels) const;
    std::unique_ptr<FactorProgram> FactorGroup(const std::vector<int>& panels, unsigned char* arena,
                                               size_t arenaBytes);
    void RunProgram(FactorProgram& pg, bool sync);
    void CheckPivots();
    // Storage of the factors: which panels stay resident, where each
    // front's G and D live, and the slots of the recomputed panels.
    void BuildLayout();

    Helmholtz& h_;
    const Analysis& an_;
    int nn_ = 0;  // nodes per panel tree
    bool layout_ = false;
    DeviceBuffer G_, D_;
    std::vector<int64_t> gOff_, dOff_;    // per (panel, node): offset in its panel's storage
    std::vector<cpx<R>*> gPtr_, dPtr_;     // per (panel, node): where G and D live
    std::vector<char> resident_;           // per panel
    std::vector<char> owned_;              // per panel: inside the handle's panel range
    std::vector<FactorFront<R>> fronts_;   // per (panel, node), transient pointers unset
    // Recomputed panels: one slot per class for G and D, the arena of their
    // factorization transients, their programs and what each slot holds.
    DeviceBuffer slotG_[3], slotD_[3], rarena_;
    std::vector<std::unique_ptr<FactorProgram>> recompute_;  // per panel (null when resident)
    int slotHolds_[3] = {-1, -1, -1};
    int64_t refactors_ = 0;
    bool AllResident() const {
        for (size_t p = 0; p < resident_.size(); ++p)
            if (owned_[p] && !resident_[p]) return false;
        return true;
    }
    std::vector<std::vector<int>> depthNodes_;
    DeviceBuffer status_;
    // One way to run the solve GEMM of one depth and direction: the kernel
    // (tensor cores, tiles of kTcRows rows; or CUDA cores, kSweepRows rows)
    // and the K-chunk of its tiles.
    struct SweepVariant {
        bool tc = false;
        int cols = kSweepCols;  // right-hand sides per tile (tensor cores: 16 or 32)
        int chunk = 0;
        size_t tiles = 0;  // arena offset of the tile list
        int n = 0;
    };
    // Per tree depth and direction: the candidate variants and the one in
    // use (complex single: chosen by timing them all, Autotune).
    struct ClassPlan {
        size_t pre = 0;
        int preN = 0;
        std::vector<size_t> bGather;
        std::vector<int> bGatherN;
        std::vector<std::vector<SweepVariant>> fVar, bVar;
        std::vector<int> fSel, bSel;
        std::vector<double> fFlops, fBytes, bFlops, bBytes;
        const SweepVariant& F(int d) const { return fVar[d][fSel[d]]; }
        const SweepVariant& B(int d) const { return bVar[d][bSel[d]]; }
    };
    // Task lists and work vectors of the panel solves for one RHS block width.
    // Plans live as long as the factors: captured sweep graphs point into them.
    struct SolvePlan {
        int k = 0;
        DeviceBuffer Rb, Y, Z, Xnd, partials, counters;
        TaskArena arena;
        ClassPlan cplan[3];
        std::vector<size_t> panelFronts;
        // complex single: the tensor-core sweep's TMA maps, two per front
        struct alignas(64) MapPair { unsigned char b[kSweepTcMapBytes]; };
        std::vector<MapPair> mapsHost;
        DeviceBuffer maps;
    };
    std::vector<std::unique_ptr<SolvePlan>> plans_;
    SolvePlan& Plan(int k);
    // Times every candidate variant of every depth of one panel solve per
    // class (scratch right-hand sides; without room for them the default
    // tiling stays) and keeps the fastest per depth and direction.  Events
    // bracket each solve-GEMM launch while tune_ is set.
    // Returns false when it measured nothing (no room for its scratch).
    bool Autotune(SolvePlan& P);
    struct TuneEvents {
        std::vector<cudaEvent_t> ev;
        int used = 0;
    };
    TuneEvents* tune_ = nullptr;
    void TuneMark() {
        if (tune_ && tune_->used < (int)tune_->ev.size())
            CUDA_CHECK(cudaEventRecord(tune_->ev[tune_->used++], h_.stream_));
    }
    bool tc_ = false;  // tensor-core sweep kernels (complex single only)
    bool factorTc_ = false;  // tensor-core factorization GEMMs (complex single only)
    // Ops of at least this many rows and K columns take tensor-core tiles.
    bool UseGemmTc(const GemmOp<R>& op) const { return factorTc_ && op.M >= 64 && op.K >= 16; }
};

template <typename R>
int64_t FactorStore<R>::TransientBytes(const std::vector<int>& panels) const {
    const PanelGeometry& g = an_.geom;
    const size_t nd = depthNodes_.size();
    std::vector<int64_t> L(nd, 0), U(nd, 0), T(nd, 0);
    for (size_t d = 0; d < nd; ++d)
        for (int p : panels) {
            const ClassStructure& cs = an_.cls[g.Class(p)];
            for (int t : depthNodes_[d]) {
                const int64_t s = cs.size[t], u = cs.usize[t];
                L[d] += (s + u) * s;
                U[d] += u * u;
                T[d] += (s / 2 + 1) * (s / 2 + 1) * 2;
            }
        }
    int64_t ua = 0, ub = 0, lm = 0, tm = 0;
    for (size_t d = 0; d < nd; ++d) {
        (d % 2 ? ub : ua) = std::max(d % 2 ? ub : ua, U[d]);
        lm = std::max(lm, L[d]);
        tm = std::max(tm, T[d]);
    }
    return (ua + ub + lm + tm) * (int64_t)sizeof(cpx<R>);
}

// Environment integer, or `dflt` when unset or not a number.
static long long EnvInt(const char* name, long long dflt) {
    const char* v = std::getenv(name);
    if (!v || !*v) return dflt;
    char* end = nullptr;
    const long long x = std::strtoll(v, &end, 10);
    return (end && *end == 0) ? x : dflt;
}

template <typename R>
void FactorStore<R>::BuildLayout() {
    const PanelGeometry& g = an_.geom;
    const XYTree& tree = an_.tree;
    nn_ = (int)tree.nodes.size();
    const int np = g.numPanels;
    depthNodes_.assign(tree.maxDepth + 1, {});
    for (int t = 0; t < nn_; ++t) depthNodes_[tree.nodes[t].depth].push_back(t);

    // per-panel storage: G then D of every front, offsets inside the panel
    gOff_.assign((size_t)np * nn_, 0);
    dOff_.assign((size_t)np * nn_, 0);
    std::vector<int64_t> gPanel(np, 0), dPanel(np, 0);
    for (int p = 0; p < np; ++p) {
        const ClassStructure& cs = an_.cls[g.Class(p)];
        for (int t = 0; t < nn_; ++t) {
            gOff_[(size_t)p * nn_ + t] = gPanel[p];
            dOff_[(size_t)p * nn_ + t] = dPanel[p];
            gPanel[p] += (int64_t)GLeadingDim(cs.size[t], cs.usize[t]) * cs.size[t];
            dPanel[p] += cs.size[t];
        }
    }
    auto panelBytes = [&](int p) { return (gPanel[p] + dPanel[p]) * (int64_t)sizeof(cpx<R>); };

    // Which panels stay resident.  The factors of all panels are kept when
    // they fit beside a reserve for the solve (the GMRES workspace of
    // PSP_B200_SOLVE_RESERVE_RHS right-hand sides at restart 20, default
    // 16) and a margin; otherwise the top panel (the costliest to factor)
    // and the lowest others are kept and the rest are recomputed into one
    // slot per class whenever a sweep reaches them (the highest panels: the
    // last one the forward sweep recomputes is the first the backward sweep
    // needs, so the slot still holds it).  PSP_B200_RESIDENT_PANELS caps the
    // resident count (0: every panel recomputed).
    size_t freeB = 0, totalB = 0;
    CUDA_CHECK(cudaMemGetInfo(&freeB, &totalB));
    const double avail = (double)freeB + (double)h_.ScratchBytes();
    const double reserveRhs = (double)EnvInt("PSP_B200_SOLVE_RESERVE_RHS", 16);
    const double reserve = reserveRhs * (double)h_.NumUnknowns() * sizeof(z64) * 25 + 1.0e9 + 0.02 * totalB;
    const long long cap = EnvInt("PSP_B200_RESIDENT_PANELS", -1);
    // panels of the handle's range only (a z-panel pipeline rank): the
    // others have no factors here
    owned_.assign(np, 0);
    for (int p = std::max(0, h_.panelBegin_); p < std::min(np, h_.panelEnd_); ++p) owned_[p] = 1;
    std::vector<int> order;  // residency priority
    if (owned_[np - 1]) order.push_back(np - 1);
    for (int p = 0; p < np - 1; ++p)
        if (owned_[p]) order.push_back(p);
    resident_ = owned_;
    double all = 0;
    for (int p = 0; p < np; ++p)
        if (owned_[p]) all += (double)panelBytes(p);
    if (cap >= 0 || all > avail - reserve) {
        // room for the slots and the recompute arena of every class that
        // may lose a panel (all classes but the top panel's, unless capped
        // to nothing), then panels in priority order while they fit
        double extra = 0;
        for (int c = 0; c < 3; ++c) {
            if (!an_.classUsed[c]) continue;
            std::vector<int> one;
            int64_t pb = 0;
            for (int p = 0; p < np; ++p)
                if (owned_[p] && g.Class(p) == c && (p != np - 1 || cap == 0)) {
                    if (one.empty()) one.push_back(p);
                    pb = std::max(pb, panelBytes(p));
                }
            if (one.empty()) continue;
            extra += (double)pb + (double)TransientBytes(one);
        }
        double used = 0;
        int count = 0;
        resident_.assign(np, 0);
        for (int p : order) {
            if (cap >= 0 && count >= cap) break;
            if (used + (double)panelBytes(p) > avail - reserve - extra) break;
            resident_[p] = 1;
            used += (double)panelBytes(p);
            ++count;
        }
    }
    int64_t gTot = 0, dTot = 0;
    for (int p = 0; p < np; ++p)
        if (resident_[p]) { gTot += gPanel[p]; dTot += dPanel[p]; }
    G_.Allocate(std::max<int64_t>(gTot, 1) * sizeof(cpx<R>));
    D_.Allocate(std::max<int64_t>(dTot, 1) * sizeof(cpx<R>));
    CUDA_CHECK(cudaMemsetAsync(G_.p, 0, G_.bytes, h_.stream_));
    std::vector<int64_t> gBase(np, 0), dBase(np, 0);
    {
        int64_t gb = 0, db = 0;
        for (int p = 0; p < np; ++p)
            if (resident_[p]) { gBase[p] = gb; dBase[p] = db; gb += gPanel[p]; db += dPanel[p]; }
    }
    int64_t slotBytesG[3] = {0, 0, 0}, slotBytesD[3] = {0, 0, 0};
    std::vector<int> recomputed[3];
    for (int p = 0; p < np; ++p)
        if (owned_[p] && !resident_[p]) {
            const int c = g.Class(p);
            slotBytesG[c] = std::max(slotBytesG[c], gPanel[p]);
            slotBytesD[c] = std::max(slotBytesD[c], dPanel[p]);
            recomputed[c].push_back(p);
        }
    int64_t rarenaBytes = 0;
    for (int c = 0; c < 3; ++c) {
        if (recomputed[c].empty()) continue;
        slotG_[c].Allocate(slotBytesG[c] * sizeof(cpx<R>));
        slotD_[c].Allocate(slotBytesD[c] * sizeof(cpx<R>));
        CUDA_CHECK(cudaMemsetAsync(slotG_[c].p, 0, slotG_[c].bytes, h_.stream_));
        rarenaBytes = std::max(rarenaBytes, TransientBytes({recomputed[c][0]}));
    }
    if (rarenaBytes) rarena_.Allocate(rarenaBytes);
    gPtr_.assign((size_t)np * nn_, nullptr);
    dPtr_.assign((size_t)np * nn_, nullptr);
    for (int p = 0; p < np; ++p) {
        const int c = g.Class(p);
        if (!owned_[p]) continue;
        cpx<R>* gp = resident_[p] ? G_.as<cpx<R>>() + gBase[p] : slotG_[c].template as<cpx<R>>();
        cpx<R>* dp = resident_[p] ? D_.as<cpx<R>>() + dBase[p] : slotD_[c].template as<cpx<R>>();
        for (int t = 0; t < nn_; ++t) {
            gPtr_[(size_t)p * nn_ + t] = gp + gOff_[(size_t)p * nn_ + t];
            dPtr_[(size_t)p * nn_ + t] = dp + dOff_[(size_t)p * nn_ + t];
        }
    }
    status_.Allocate(sizeof(int));
    CUDA_CHECK(cudaMemsetAsync(status_.p, 0, sizeof(int), h_.stream_));

    fronts_.assign((size_t)np * nn_, FactorFront<R>());
    for (int p = 0; p < np; ++p) {
        const int c = g.Class(p);
        const ClassStructure& cs = an_.cls[c];
        for (int t = 0; t < nn_; ++t) {
            FactorFront<R>& f = fronts_[(size_t)p * nn_ + t];
            std::memset(&f, 0, sizeof(f));
            f.G = gPtr_[(size_t)p * nn_ + t];
            f.D = dPtr_[(size_t)p * nn_ + t];
            f.rel = h_.dRel_[c].as<int>() + cs.lowerOff[t];
            f.s = cs.size[t];
            f.u = cs.usize[t];
            f.ldg = GLeadingDim(f.s, f.u);
            f.parent = tree.nodes[t].parent < 0 ? -1 : p * nn_ + tree.nodes[t].parent;
            f.cls = c;
            f.ndOff = cs.off[t];
            f.vOffset = g.SubVOffset(p);
            f.s3aOff = h_.s3aOff_[p];
        }
    }
    // recomputed panels: one program each, transients in the recompute arena
    recompute_.clear();
    recompute_.resize(np);
    for (int p = 0; p < np; ++p)
        if (owned_[p] && !resident_[p])
            recompute_[p] = FactorGroup({p}, rarena_.template as<unsigned char>(), rarena_.bytes);
    layout_ = true;
}

template <typename R>
void FactorStore<R>::Factor() {
    if (!layout_) BuildLayout();
    CUDA_CHECK(cudaMemsetAsync(status_.p, 0, sizeof(int), h_.stream_));
    for (int& c : slotHolds_) c = -1;  // the velocity changed: slots are stale
    refactors_ = 0;
    // replay the recorded factorization while the scratch has not moved
    bool replay = !program_.empty();
    for (const auto& pg : program_)
        replay = replay && pg->arena == h_.Scratch(0) && pg->arenaBytes <= h_.ScratchBytes();
    if (!replay) {
        program_.clear();
        const PanelGeometry& g = an_.geom;
        std::vector<int> res;
        for (int p = 0; p < g.numPanels; ++p)
            if (resident_[p]) res.push_back(p);
        // groups of resident panels whose transients fit in 80% of the free
        // memory (the scratch counts as free: it is reused)
        size_t freeB = 0, totalB = 0;
        CUDA_CHECK(cudaMemGetInfo(&freeB, &totalB));
        const int64_t budget = (int64_t)(0.8 * ((double)freeB + (double)h_.ScratchBytes()));
        int groupSize = std::max<int>(1, (int)res.size());
        auto slice = [&](size_t i0, int n) {
            return std::vector<int>(res.begin() + i0, res.begin() + std::min(res.size(), i0 + n));
        };
        auto maxTransient = [&](int n) {
            int64_t m = 0;
            for (size_t i0 = 0; i0 < res.size(); i0 += n) m = std::max(m, TransientBytes(slice(i0, n)));
            return m;
        };
        while (groupSize > 1 && maxTransient(groupSize) > budget) groupSize = (groupSize + 1) / 2;
        const int64_t need = res.empty() ? 0 : maxTransient(groupSize);
        unsigned char* arena = static_cast<unsigned char*>(h_.Scratch(need));
        for (size_t i0 = 0; i0 < res.size(); i0 += groupSize)
            program_.push_back(FactorGroup(slice(i0, groupSize), arena, need));
    }
    for (auto& pg : program_) RunProgram(*pg, false);
    CUDA_CHECK(cudaStreamSynchronize(h_.stream_));
    CheckPivots();
}

template <typename R>
void FactorStore<R>::EnsurePanel(int p) {
    if (resident_[p]) return;
    const int c = an_.geom.Class(p);
    if (slotHolds_[c] == p) return;
    RunProgram(*recompute_[p], false);
    slotHolds_[c] = p;
    ++refactors_;
}

template <typename R>
void FactorStore<R>::CheckPivots() {
    int st = 0;
    CUDA_CHECK(cudaMemcpyAsync(&st, status_.p, sizeof(int), cudaMemcpyDeviceToHost, h_.stream_));
    CUDA_CHECK(cudaStreamSynchronize(h_.stream_));
    if (st & 1) throw PspError(kRuntimeError, "zero or non-finite pivot in a panel factorization");
    if (st & 2) throw PspError(kRuntimeError, "a tensor-core pipeline wait timed out in the factorization");
}

template <typename R>
std::unique_ptr<typename FactorStore<R>::FactorProgram> FactorStore<R>::FactorGroup(const std::vector<int>& panels,
                                                                                   unsigned char* arenaBase,
                                                                                   size_t arenaBytes) {
    const PanelGeometry& g = an_.geom;
    const XYTree& tree = an_.tree;
    const int nd = (int)depthNodes_.size();
    const int ng = (int)panels.size();
    cudaStream_t st = h_.stream_;
    // per-depth transient layout
    std::vector<int64_t> Lsz(nd, 0), Usz(nd, 0), Tsz(nd, 0);
    std::vector<int64_t> Lpos((size_t)ng * nn_), Upos((size_t)ng * nn_), Tpos((size_t)ng * nn_);
    for (int d = 0; d < nd; ++d)
        for (int gi = 0; gi < ng; ++gi) {
            const ClassStructure& cs = an_.cls[g.Class(panels[gi])];
            for (int t : depthNodes_[d]) {
                const int64_t s = cs.size[t], u = cs.usize[t];
                const size_t i = (size_t)gi * nn_ + t;
                Lpos[i] = Lsz[d]; Lsz[d] += (s + u) * s;
                Upos[i] = Usz[d]; Usz[d] += u * u;
                Tpos[i] = Tsz[d]; Tsz[d] += (s / 2 + 1) * (s / 2 + 1) * 2;
            }
        }
    int64_t ua = 0, ub = 0, lm = 0, tm = 0;
    for (int d = 0; d < nd; ++d) {
        if (d % 2) ub = std::max(ub, Usz[d]); else ua = std::max(ua, Usz[d]);
        lm = std::max(lm, Lsz[d]);
        tm = std::max(tm, Tsz[d]);
    }
    if ((size_t)(ua + ub + lm + tm) * sizeof(cpx<R>) > arenaBytes)
        throw PspError(kRuntimeError, "factorization transients exceed their arena");
    std::unique_ptr<FactorProgram> pgHolder(new FactorProgram);
    FactorProgram& pg = *pgHolder;
    pg.arena = arenaBase;
    pg.arenaBytes = arenaBytes;
    cpx<R>* UA = reinterpret_cast<cpx<R>*>(arenaBase);
    cpx<R>* UB = UA + ua;
    cpx<R>* Lb = UB + ub;
    cpx<R>* Tb = Lb + lm;
    // the group's fronts, indexed gi * nn_ + t (parents likewise)
    std::vector<FactorFront<R>> all((size_t)ng * nn_);
    for (int gi = 0; gi < ng; ++gi)
        for (int t = 0; t < nn_; ++t) {
            FactorFront<R>& f = all[(size_t)gi * nn_ + t];
            f = fronts_[(size_t)panels[gi] * nn_ + t];
            f.parent = tree.nodes[t].parent < 0 ? -1 : gi * nn_ + tree.nodes[t].parent;
        }
    for (int d = 0; d < nd; ++d)
        for (int gi = 0; gi < ng; ++gi)
            for (int t : depthNodes_[d]) {
                const size_t i = (size_t)gi * nn_ + t;
                FactorFront<R>& f = all[i];
                f.L = Lb + Lpos[i];
                f.U = (d % 2 ? UB : UA) + Upos[i];
                f.T = Tb + Tpos[i];
            }
    const char* arenaP = reinterpret_cast<const char*>(arenaBase);

    TaskArena& arenaTasks = pg.tasks;
    pg.frontsOff = arenaTasks.Push(all);
    std::vector<Step>& steps = pg.steps;
    std::vector<GemmOp<R>> ops;
    std::vector<GemmTile> tiles;
    std::vector<GemmTcTile> tilesTc;
    auto pushGemm = [&]() {
        if (tiles.empty() && tilesTc.empty()) { ops.clear(); return; }
        Step s;
        s.kind = Step::kGemm;
        for (const GemmOp<R>& op : ops) OpCost(op, s.flops, s.abytes);
        s.a = arenaTasks.Push(ops);
        if (!tiles.empty()) s.b = arenaTasks.Push(tiles);
        if (!tilesTc.empty()) s.c = arenaTasks.Push(tilesTc);
        s.n = (int)tiles.size();
        s.nTc = (int)tilesTc.size();
        steps.push_back(s);
        ops.clear();
        tiles.clear();
        tilesTc.clear();
    };
    // Tiles of `op` (index i) for the tensor-core or the CUDA-core kernel.
    auto route = [&](const GemmOp<R>& op, int i, std::vector<GemmTile>& cc, std::vector<GemmTcTile>& tc) {
        if constexpr (std::is_same<R, float>::value) {
            if (UseGemmTc(op) && GemmTcEligible(op)) {
                AppendGemmTilesTc(op, tc);
                return;
            }
        }
        AppendGemmTiles(op, i, kGemmSquare, cc);
    };
    auto addOp = [&](const GemmOp<R>& op) {
        route(op, (int)ops.size(), tiles, tilesTc);
        ops.push_back(op);
    };
    const R one = 1, mone = -1, zero = 0;
    for (int d = nd - 1; d >= 0; --d) {
        std::vector<int> list;
        int maxS = 0;
        for (int gi = 0; gi < ng; ++gi)
            for (int t : depthNodes_[d]) {
                list.push_back(gi * nn_ + t);
                maxS = std::max(maxS, all[(size_t)gi * nn_ + t].s);
            }
        if (list.empty()) continue;
        // zero this depth's frontal columns and update matrices
        {
            Step s;
            s.kind = Step::kMemset;
            s.a = (size_t)((const char*)Lb - arenaP);
            s.bytes = Lsz[d] * sizeof(cpx<R>);
            steps.push_back(s);
            s.a = (size_t)((const char*)(d % 2 ? UB : UA) - arenaP);
            s.bytes = Usz[d] * sizeof(cpx<R>);
            steps.push_back(s);
        }
        {
            Step s;
            s.kind = Step::kAssemble;
            s.a = arenaTasks.Push(list);
            s.n = (int)list.size();
            steps.push_back(s);
        }
        for (int slot = 0; slot < 2; ++slot) {
            std::vector<int2> ext;
            for (int fi : list) {
                const int t = fi % nn_, p = fi / nn_;
                const XYNode& node = tree.nodes[t];
                if (node.numChildren <= slot) continue;
                const int ci = p * nn_ + node.child[slot];
                for (int b0 = 0; b0 < all[ci].u; b0 += 32) ext.push_back(make_int2(ci, b0));
            }
            if (ext.empty()) continue;
            Step s;
            s.kind = Step::kExtend;
            s.a = arenaTasks.Push(ext);
            s.n = (int)ext.size();
            steps.push_back(s);
        }
        // right-looking blocked LDL^T over the pivot columns
        for (int J = 0; J < maxS; J += kNB) {
            std::vector<int> dl;
            std::vector<int2> tr;
            for (int fi : list) {
                const FactorFront<R>& f = all[fi];
                if (f.s <= J) continue;
                dl.push_back(fi);
                const int b = std::min(kNB, f.s - J);
                for (int r0 = J + b; r0 < f.s + f.u; r0 += kTrsmRows) tr.push_back(make_int2(fi, r0));
                const int M = f.s + f.u - J - b, N = f.s - J - b;
                if (M > 0 && N > 0) {
                    const int64_t ld = f.s + f.u;
                    GemmOp<R> op = MakeOp<R>(f.L + (J + b) + J * ld, ld, 0, f.L + (J + b) + J * ld, ld, 1,
                                             f.L + (J + b) + (J + b) * ld, ld, M, N, b, mone, one);
                    op.d = f.D + J;
                    op.lowerC = 1;
                    addOp(op);
                }
            }
            Step s;
            s.kind = Step::kDiag;
            s.a = arenaTasks.Push(dl);
            s.n = (int)dl.size();
            s.J = J;
            steps.push_back(s);
            if (!tr.empty()) {
                Step t;
                t.kind = Step::kTrsm;
                t.a = arenaTasks.Push(tr);
                t.n = (int)tr.size();
                t.J = J;
                steps.push_back(t);
            }
            pushGemm();
        }
        // inv(L11) by recursive doubling of the kNB diagonal inverses
        for (int S = kNB; S < maxS; S *= 2) {
            std::vector<GemmOp<R>> ops2;
            std::vector<GemmTile> tiles2;
            std::vector<GemmTcTile> tilesTc2;
            for (int fi : list) {
                const FactorFront<R>& f = all[fi];
                const int64_t ld = f.s + f.u;
                int64_t toff = 0;
                for (int a0 = 0; a0 + S < f.s; a0 += 2 * S) {
                    const int a1 = a0 + S, a2 = std::min(a0 + 2 * S, f.s);
                    const int m = a2 - a1, n = a1 - a0;
                    cpx<R>* T = f.T + toff;
                    toff += (int64_t)m * n;
                    const int64_t lg = f.ldg;
                    GemmOp<R> op1 = MakeOp<R>(f.L + a1 + a0 * ld, ld, 0, f.G + a0 + a0 * lg, lg, 0, T, m, m, n, n,
                                              one, zero);
                    op1.triB = 1;
                    addOp(op1);
                    GemmOp<R> op2 = MakeOp<R>(f.G + a1 + a1 * lg, lg, 0, T, m, 0, f.G + a1 + a0 * lg, lg, m, n, m,
                                              mone, zero);
                    op2.triA = 1;
                    route(op2, (int)ops2.size(), tiles2, tilesTc2);
                    ops2.push_back(op2);
                }
            }
            pushGemm();
            ops = ops2;
            tiles = tiles2;
            tilesTc = tilesTc2;
            pushGemm();
        }
        // G21 = -L21 inv(L11) and the Schur complement U -= L21 D L21^T
        for (int fi : list) {
            const FactorFront<R>& f = all[fi];
            if (f.u == 0) continue;
            const int64_t ld = f.s + f.u;
            GemmOp<R> g21 = MakeOp<R>(f.L + f.s, ld, 0, f.G, f.ldg, 0, f.G + f.s, f.ldg, f.u, f.s, f.s, mone, zero);
            g21.triB = 1;
            addOp(g21);
            GemmOp<R> sch = MakeOp<R>(f.L + f.s, ld, 0, f.L + f.s, ld, 1, f.U, f.u, f.u, f.u, f.s, mone, one);
            sch.d = f.D;
            sch.lowerC = 1;
            addOp(sch);
        }
        pushGemm();
    }
    arenaTasks.Upload(st);
    return pgHolder;
}

template <typename R>
void FactorStore<R>::RunProgram(FactorProgram& pg, bool sync) {
    cudaStream_t st = h_.stream_;
    const TaskArena& arenaTasks = pg.tasks;
    const FactorFront<R>* dFronts = arenaTasks.template At<FactorFront<R>>(pg.frontsOff);
    for (const Step& s : pg.steps) {
        switch (s.kind) {
            case Step::kMemset:
                if (s.bytes) CUDA_CHECK(cudaMemsetAsync(pg.arena + s.a, 0, s.bytes, st));
                break;
            case Step::kAssemble: {
                ProfScope ps(st, kProfAssemble);
                LaunchAssemble<R>(dFronts, arenaTasks.At<int>(s.a), s.n, h_.ap_, st);
                break;
            }
            case Step::kExtend: {
                ProfScope ps(st, kProfExtendAdd);
                LaunchExtendAdd<R>(dFronts, arenaTasks.At<int2>(s.a), s.n, st);
                break;
            }
            case Step::kDiag: {
                ProfScope ps(st, kProfLdlDiag);
                LaunchLdlDiag<R>(dFronts, arenaTasks.At<int>(s.a), s.n, s.J, status_.as<int>(), st);
                break;
            }
            case Step::kTrsm: {
                ProfScope ps(st, kProfLdlTrsm);
                LaunchLdlTrsm<R>(dFronts, arenaTasks.At<int2>(s.a), s.n, s.J, st);
                break;
            }
            case Step::kGemm: {
                ProfScope ps(st, kProfFactorGemm, s.flops, s.abytes);
                const GemmOp<R>* ops = arenaTasks.At<GemmOp<R>>(s.a);
                if (s.n) LaunchGemm<R>(ops, arenaTasks.At<GemmTile>(s.b), s.n, kGemmSquare, st);
                if constexpr (std::is_same<R, float>::value) {
                    if (s.nTc) LaunchGemmTc(arenaTasks.At<GemmTcTile>(s.c), s.nTc, status_.as<int>(), st);
                }
                break;
            }
        }
    }
    if (sync) CUDA_CHECK(cudaStreamSynchronize(st));
}

template <typename R>
typename FactorStore<R>::SolvePlan& FactorStore<R>::Plan(int k) {
    for (auto& pl : plans_)
        if (pl->k == k) return *pl;
    plans_.emplace_back(new SolvePlan);
    SolvePlan& P = *plans_.back();
    P.k = k;
    const PanelGeometry& g = an_.geom;
    const XYTree& tree = an_.tree;
    const int np = g.numPanels;
    const int nd = (int)depthNodes_.size();
    // Work vectors per class: R planes (3 (s+u) k), Y (s k) and Z ((s+u) k).
    std::vector<std::vector<int64_t>> rOff(3), yOff(3), zOff(3);
    int64_t maxR = 0, maxY = 0, maxZ = 0;
    int maxSub = 0;
    for (int c = 0; c < 3; ++c) {
        if (!an_.classUsed[c]) continue;
        const ClassStructure& cs = an_.cls[c];
        rOff[c].resize(nn_); yOff[c].resize(nn_); zOff[c].resize(nn_);
        int64_t tr = 0, ty = 0, tz = 0;
        for (int t = 0; t < nn_; ++t) {
            rOff[c][t] = tr; yOff[c][t] = ty; zOff[c][t] = tz;
            tr += (int64_t)(cs.size[t] + cs.usize[t]) * 3 * k;
            ty += (int64_t)cs.size[t] * k;
            tz += (int64_t)(cs.size[t] + cs.usize[t]) * k;
        }
        maxR = std::max(maxR, tr); maxY = std::max(maxY, ty); maxZ = std::max(maxZ, tz);
        maxSub = std::max(maxSub, cs.nSub);
    }
    P.Rb.Allocate(maxR * sizeof(cpx<R>));
    P.Y.Allocate(maxY * sizeof(cpx<R>));
    P.Z.Allocate(maxZ * sizeof(cpx<R>));
    P.Xnd.Allocate((size_t)maxSub * k * sizeof(cpx<R>));
    P.arena.host.clear();
    P.panelFronts.assign(np, 0);
    if (tc_) {
        P.mapsHost.assign((size_t)np * nn_, {});
        P.maps.Allocate(P.mapsHost.size() * sizeof(typename SolvePlan::MapPair));
    }
    for (int p = 0; p < np; ++p) {
        const int c = g.Class(p);
        const ClassStructure& cs = an_.cls[c];
        std::vector<SweepFront<R>> fr(nn_);
        for (int t = 0; t < nn_; ++t) {
            SweepFront<R>& f = fr[t];
            const XYNode& node = tree.nodes[t];
            f.G = gPtr_[(size_t)p * nn_ + t];
            f.D = dPtr_[(size_t)p * nn_ + t];
            f.Rb = P.Rb.template as<cpx<R>>() + rOff[c][t];
            f.parentRb = node.parent >= 0 ? P.Rb.template as<cpx<R>>() + rOff[c][node.parent] : nullptr;
            f.Y = P.Y.template as<cpx<R>>() + yOff[c][t];
            f.Z = P.Z.template as<cpx<R>>() + zOff[c][t];
            f.lower = h_.dLower_[c].as<int>() + cs.lowerOff[t];
            f.rel = h_.dRel_[c].as<int>() + cs.lowerOff[t];
            f.s = cs.size[t];
            f.u = cs.usize[t];
            f.ndOff = cs.off[t];
            f.childSlot = (node.parent >= 0 && tree.nodes[node.parent].child[1] == t) ? 1 : 0;
            f.ldg = GLeadingDim(f.s, f.u);
            f.tmap = nullptr;
            if constexpr (std::is_same<R, float>::value) {
                if (tc_ && f.s > 0 && owned_[p]) {
                    const size_t i = (size_t)p * nn_ + t;
                    EncodeSweepTcMaps(f, P.mapsHost[i].b);
                    f.tmap = P.maps.template as<unsigned char>() + i * sizeof(typename SolvePlan::MapPair);
                }
            }
        }
        P.panelFronts[p] = P.arena.Push(fr);
    }
    // Tiles of one depth and direction: rows of a tile share one K range
    // (inv(L11) is triangular, so the forward range stops at the tile's last
    // row and the backward range starts at its first), split into chunks.
    // The default chunk starts at the kernel's longest (the tensor-core
    // kernels are persistent and pipeline across tiles, so long chunks cost
    // nothing extra and save split-K partial sums) and only shrinks to give
    // every SM tiles; `forceChunk` > 0 fixes it instead (tuning candidates).
    int64_t maxPartialRows = kTcRows, maxCounters = 1;
    // Longest K-chunk of a tensor-core tile (PSP_B200_SWEEP_TC_MAX_CHUNK),
    // and a fixed chunk for the default tensor-core tiling in place of the
    // shrinking rule below (PSP_B200_SWEEP_TC_CHUNK, tests; 0 = unset).
    // Both are rounded down to a power of two from 16 to 512: a backward
    // tile's K start is the innermost coordinate of its TMA copies, which
    // must be even (16-byte aligned complex-single entries), and chunks of
    // whole stages keep it so.
    auto chunkSetting = [](long long v) {
        int c = 16;
        while (2LL * c <= std::min(v, 512LL)) c *= 2;
        return c;
    };
    const int tcMaxChunk = chunkSetting(EnvInt("PSP_B200_SWEEP_TC_MAX_CHUNK", 512));
    const long long tcChunkEnv = EnvInt("PSP_B200_SWEEP_TC_CHUNK", 0);
    const int tcFixedChunk = tcChunkEnv > 0 ? std::min(tcMaxChunk, chunkSetting(tcChunkEnv)) : 0;
    auto makeTiles = [&](const ClassStructure& cs, int d, bool fwd, bool tcTiles, int cols, int forceChunk,
                         std::vector<SweepTile>& tiles) {
        const int maxChunk = tcTiles ? tcMaxChunk : SweepMaxChunk<R>();
        if (forceChunk > maxChunk) forceChunk = maxChunk;
        const int tileRows = tcTiles ? kTcRows : kSweepRows;
        const int subs = cols / kSweepCols;  // partial slots and counters per split tile
        auto build = [&](int kc, bool emit) {
            int64_t n = 0, slots = 0, counters = 0;
            for (int t : depthNodes_[d]) {
                const int s = cs.size[t], u = cs.usize[t];
                const int M = fwd ? s + u : s, K = fwd ? s : s + u;
                for (int col0 = 0; col0 < k; col0 += cols)
                    for (int row0 = 0; row0 < M; row0 += tileRows) {
                        const int kb = fwd ? 0 : row0;
                        const int ke = fwd ? std::min(K, row0 + tileRows) : K;
                        const int ns = std::max(1, (int)CeilDiv(ke - kb, kc));
                        for (int sp = 0; sp < ns; ++sp) {
                            if (emit) {
                                SweepTile tl;
                                tl.front = t; tl.row0 = row0; tl.col0 = col0;
                                tl.k0 = kb + sp * kc;
                                tl.k1 = std::min(ke, kb + (sp + 1) * kc);
                                tl.split = sp; tl.nsplit = ns;
                                tl.slot = ns > 1 ? (int)slots : -1;
                                tl.counter = ns > 1 ? (int)counters : -1;
                                tiles.push_back(tl);
                            }
                            ++n;
                        }
                        if (ns > 1) { slots += ns; ++counters; }
                    }
            }
            if (emit) {
                maxPartialRows = std::max(maxPartialRows, slots * tileRows * subs);
                maxCounters = std::max(maxCounters, counters * subs);
            }
            return n;
        };
        // default: shrink until the launch has tiles for every SM (CUDA-core
        // CTAs, two per SM) or for half of them (persistent tensor-core CTAs,
        // whose long K pipelines beat extra split-K partial sums)
        const int64_t minTiles = tcTiles ? 74 : 2 * 148;
        int kc = forceChunk > 0 ? forceChunk : maxChunk;
        while (forceChunk <= 0 && kc > 64 && build(kc, false) < minTiles) kc /= 2;
        build(kc, true);
        // longest K ranges first, so the launch does not end on a long tail
        std::stable_sort(tiles.begin(), tiles.end(), [](const SweepTile& a, const SweepTile& b) {
            return (a.k1 - a.k0) > (b.k1 - b.k0);
        });
        return kc;
    };
    auto depthCost = [&](const ClassStructure& cs, int d, bool fwd, double& flops, double& bytes) {
        for (int t : depthNodes_[d]) {
            const double s = cs.size[t], u = cs.usize[t];
            const double nz = (s + u) * s - s * (s - 1) / 2;  // nonzeros of G
            flops += 8.0 * nz * k;
            bytes += sizeof(cpx<R>) * (nz + (fwd ? (s + 2 * (s + u)) : (2 * (s + u) + 2 * s)) * k);
        }
    };
    // Candidates of one depth and direction: the default tiling of each
    // kernel and, with tensor cores, the other chunk lengths (a tiling equal
    // to an earlier candidate's is skipped).
    // With more than 16 right-hand sides the tensor-core tiles take 32 of
    // them (one split of each G stage for twice the columns); the 16-wide
    // default stays a candidate.
    auto makeVariants = [&](const ClassStructure& cs, int d, bool fwd, std::vector<SweepVariant>& out) {
        struct Cand { bool tc; int cols, chunk; };
        std::vector<Cand> cand;
        if (tc_) {
            const int wide = k > kSweepCols ? 32 : kSweepCols;
            cand.push_back({true, wide, tcFixedChunk});
            for (int kc : {64, 128, 256, 512}) cand.push_back({true, wide, kc});
            if (wide != kSweepCols)
                for (int kc : {0, 512}) cand.push_back({true, kSweepCols, kc});
            cand.push_back({false, kSweepCols, 0});
            for (int kc : {64, 128}) cand.push_back({false, kSweepCols, kc});
        } else {
            cand.push_back({false, kSweepCols, 0});
        }
        std::vector<std::vector<SweepTile>> seen;
        for (const auto& cd : cand) {
            std::vector<SweepTile> tiles;
            SweepVariant v;
            v.tc = cd.tc;
            v.cols = cd.cols;
            v.chunk = makeTiles(cs, d, fwd, cd.tc, cd.cols, cd.chunk, tiles);
            bool dup = false;
            for (size_t i = 0; i < seen.size() && !dup; ++i)
                dup = out[i].tc == v.tc && out[i].cols == v.cols && seen[i].size() == tiles.size() &&
                      std::equal(tiles.begin(), tiles.end(), seen[i].begin(), [](const SweepTile& a, const SweepTile& b) {
                          return a.front == b.front && a.row0 == b.row0 && a.col0 == b.col0 && a.k0 == b.k0 &&
                                 a.k1 == b.k1;
                      });
            if (dup) continue;
            v.tiles = P.arena.Push(tiles);
            v.n = (int)tiles.size();
            out.push_back(v);
            seen.push_back(std::move(tiles));
        }
    };
    for (int c = 0; c < 3; ++c) {
        if (!an_.classUsed[c]) continue;
        const ClassStructure& cs = an_.cls[c];
        ClassPlan& cp = P.cplan[c];
        cp.bGather.assign(nd, 0);
        cp.bGatherN.assign(nd, 0);
        cp.fVar.assign(nd, {});
        cp.bVar.assign(nd, {});
        cp.fSel.assign(nd, 0);
        cp.bSel.assign(nd, 0);
        cp.fFlops.assign(nd, 0); cp.fBytes.assign(nd, 0); cp.bFlops.assign(nd, 0); cp.bBytes.assign(nd, 0);
        std::vector<int2> pre;
        for (int d = 0; d < nd; ++d) {
            std::vector<int2> bg;
            makeVariants(cs, d, true, cp.fVar[d]);
            makeVariants(cs, d, false, cp.bVar[d]);
            depthCost(cs, d, true, cp.fFlops[d], cp.fBytes[d]);
            depthCost(cs, d, false, cp.bFlops[d], cp.bBytes[d]);
            for (int t : depthNodes_[d])
                for (int i0 = 0; i0 < cs.size[t] + cs.usize[t]; i0 += kSweepRows) {
                    bg.push_back(make_int2(t, i0));
                    pre.push_back(make_int2(t, i0));
                }
            cp.bGather[d] = P.arena.Push(bg);
            cp.bGatherN[d] = (int)bg.size();
        }
        cp.pre = P.arena.Push(pre);
        cp.preN = (int)pre.size();
    }
    P.partials.Allocate((size_t)maxPartialRows * kSweepCols * sizeof(cpx<R>));
    P.counters.Allocate((size_t)maxCounters * sizeof(int));
    CUDA_CHECK(cudaMemsetAsync(P.counters.p, 0, P.counters.bytes, h_.stream_));
    P.arena.Upload(h_.stream_);
    if (tc_) {
        CUDA_CHECK(cudaMemcpyAsync(P.maps.p, P.mapsHost.data(), P.maps.bytes, cudaMemcpyHostToDevice, h_.stream_));
        // PSP_B200_SWEEP_AUTOTUNE: unset = time every candidate per depth on
        // problems of at least 2^20 unknowns (where the timing, a few sweeps'
        // worth, is small against a solve), else the default tiling; "1" =
        // time them at any size; "0" = the default tensor-core tiling
        // everywhere; "alternate" = a fixed mix of tensor-core and CUDA-core
        // depths (tests).
        const char* env = std::getenv("PSP_B200_SWEEP_AUTOTUNE");
        std::string mode = env ? env : "";
        if (mode.empty()) mode = h_.NumUnknowns() >= (int64_t(1) << 20) ? "1" : "0";
        if (mode == "alternate") {
            for (ClassPlan& cp : P.cplan)
                for (size_t d = 0; d < cp.fVar.size(); ++d) {
                    auto firstOf = [](const std::vector<SweepVariant>& vs, bool tc) {
                        for (size_t i = 0; i < vs.size(); ++i)
                            if (vs[i].tc == tc) return (int)i;
                        return 0;
                    };
                    cp.fSel[d] = firstOf(cp.fVar[d], d % 2 == 1);
                    cp.bSel[d] = firstOf(cp.bVar[d], d % 2 == 0);
                }
        } else if (mode == "1") {
            std::string key = std::to_string(k) + "/" + std::to_string(h_.device());
            for (int c = 0; c < 3; ++c) {
                if (!an_.classUsed[c]) continue;
                const ClassStructure& cs = an_.cls[c];
                key += "|" + std::to_string(c) + ":";
                for (size_t t = 0; t < cs.size.size(); ++t)
                    key += std::to_string(cs.size[t]) + "," + std::to_string(cs.usize[t]) + ";";
            }
            std::vector<int> routes;
            auto lookup = [&] {
                std::lock_guard<std::mutex> lock(gRouteMutex);
                auto it = gRoutes.find(key);
                if (it != gRoutes.end()) routes = it->second;
            };
            lookup();
            if (routes.empty()) {
                // one tuning run at a time in the process: a handle with the
                // same structure waits for it and reuses its choices, and
                // no two tuning runs time each other's launches
                std::lock_guard<std::mutex> tuning(gTuneMutex);
                lookup();
                if (routes.empty() && Autotune(P)) {
                    // only measured choices are shared: a handle that could
                    // not time its candidates keeps the default tiling, and a
                    // later one with room tunes
                    for (const ClassPlan& cp : P.cplan) {
                        routes.insert(routes.end(), cp.fSel.begin(), cp.fSel.end());
                        routes.insert(routes.end(), cp.bSel.begin(), cp.bSel.end());
                    }
                    std::lock_guard<std::mutex> lock(gRouteMutex);
                    gRoutes.emplace(key, routes);
                }
            }
            size_t i = 0;
            for (ClassPlan& cp : P.cplan) {
                for (int& r : cp.fSel) r = routes.empty() ? 0 : routes[i++];
                for (int& r : cp.bSel) r = routes.empty() ? 0 : routes[i++];
            }
        }
    }
    return P;
}

template <typename R>
bool FactorStore<R>::Autotune(SolvePlan& P) {
    const PanelGeometry& g = an_.geom;
    const int nd = (int)depthNodes_.size(), k = P.k;
    const int reps = 2;
    DeviceBuffer scratch;
    try {
        scratch.Allocate((size_t)h_.NumUnknowns() * k * sizeof(z64));
    } catch (const PspError& e) {
        if (e.code != kOutOfMemory) throw;
        cudaGetLastError();  // no room for timing runs: keep the default tiling
        return false;
    }
    CUDA_CHECK(cudaMemsetAsync(scratch.p, 0, scratch.bytes, h_.stream_));
    TuneEvents te;
    te.ev.resize(4 * nd);
    for (cudaEvent_t& e : te.ev) CUDA_CHECK(cudaEventCreate(&e));
    const char* verbose = std::getenv("PSP_B200_SWEEP_AUTOTUNE_VERBOSE");
    const bool talk = verbose && verbose[0] == '1';
    try {
        for (int c = 0; c < 3; ++c) {
            int p = -1;
            for (int q = 0; q < g.numPanels && p < 0; ++q)
                if (g.Class(q) == c && owned_[q]) p = q;
            if (p < 0) continue;
            ClassPlan& cp = P.cplan[c];
            size_t maxVar = 0;
            for (int d = 0; d < nd; ++d) maxVar = std::max({maxVar, cp.fVar[d].size(), cp.bVar[d].size()});
            // [direction][depth][variant] best milliseconds
            std::vector<std::vector<float>> best[2];
            for (int dir = 0; dir < 2; ++dir) {
                best[dir].assign(nd, {});
                for (int d = 0; d < nd; ++d) best[dir][d].assign((dir ? cp.bVar : cp.fVar)[d].size(), 1e30f);
            }
            // run v times every depth's v-th candidate (its first where it has fewer)
            for (size_t v = 0; v < maxVar; ++v) {
                for (int d = 0; d < nd; ++d) {
                    cp.fSel[d] = v < cp.fVar[d].size() ? (int)v : 0;
                    cp.bSel[d] = v < cp.bVar[d].size() ? (int)v : 0;
                }
                for (int rep = 0; rep <= reps; ++rep) {
                    te.used = 0;
                    tune_ = &te;
                    SolvePanel(scratch.as<z64>(), k, k, p, 0, 0);
                    tune_ = nullptr;
                    CUDA_CHECK(cudaStreamSynchronize(h_.stream_));
                    if (rep == 0 || te.used != 4 * nd) continue;  // the first run warms up
                    for (int i = 0; i < nd; ++i) {
                        float fms = 0, bms = 0;
                        CUDA_CHECK(cudaEventElapsedTime(&fms, te.ev[2 * i], te.ev[2 * i + 1]));
                        CUDA_CHECK(cudaEventElapsedTime(&bms, te.ev[2 * nd + 2 * i], te.ev[2 * nd + 2 * i + 1]));
                        const int df = nd - 1 - i;  // the forward walks the depths bottom-up
                        float& bf = best[0][df][cp.fSel[df]];
                        float& bb = best[1][i][cp.bSel[i]];
                        bf = std::min(bf, fms);
                        bb = std::min(bb, bms);
                    }
                }
            }
            for (int d = 0; d < nd; ++d) {
                for (int dir = 0; dir < 2; ++dir) {
                    const std::vector<float>& b = best[dir][d];
                    (dir ? cp.bSel : cp.fSel)[d] = (int)(std::min_element(b.begin(), b.end()) - b.begin());
                }
                if (talk) {
                    std::fprintf(stderr, "sweep autotune k=%d class %d depth %2d:", k, c, d);
                    for (int dir = 0; dir < 2; ++dir) {
                        const std::vector<SweepVariant>& vs = (dir ? cp.bVar : cp.fVar)[d];
                        std::fprintf(stderr, dir ? "  bwd" : " fwd");
                        for (size_t i = 0; i < vs.size(); ++i)
                            std::fprintf(stderr, " %s%s%d/%d %.4f", (int)i == (dir ? cp.bSel : cp.fSel)[d] ? "*" : "",
                                         vs[i].tc ? "tc" : "cc", vs[i].cols, vs[i].chunk, best[dir][d][i]);
                    }
                    std::fprintf(stderr, "\n");
                }
            }
        }
    } catch (...) {
        tune_ = nullptr;
        for (cudaEvent_t e : te.ev) cudaEventDestroy(e);
        throw;
    }
    for (cudaEvent_t e : te.ev) CUDA_CHECK(cudaEventDestroy(e));
    return true;
}

template <typename R>
void FactorStore<R>::SolvePanel(z64* B, int ldk, int k, int p, int inMode, int outAcc, int zBase) {
    if (!owned_[p]) throw PspError(kLogicError, "panel " + std::to_string(p) + " is outside the handle's panel range");
    SolvePlan& P = Plan(k);
    EnsurePanel(p);
    const PanelGeometry& g = an_.geom;
    const int c = g.Class(p);
    const ClassPlan& cp = P.cplan[c];
    cudaStream_t st = h_.stream_;
    PanelIO io;
    io.ndToNat = h_.dNdToNat_[c].as<int>();
    io.nx = an_.disc.nx;
    io.nxy = an_.disc.nx * an_.disc.ny;
    io.nz = an_.disc.nz - zBase;  // kernels index plane nz - 1 - v: relative to the slab's first plane
    io.ldk = ldk;
    io.padding = g.Padding(p);
    io.vOffset = g.SubVOffset(p);
    io.lowV = g.LowV(p);
    io.highV = g.LowV(p) + g.Depth(p) - 1;
    io.inMode = inMode;
    io.outAccumulate = outAcc;
    io.sp = h_.sp_;
    const SweepFront<R>* fr = P.arena.template At<SweepFront<R>>(P.panelFronts[p]);
    SweepWork w;
    w.partials = P.partials.p;
    w.counters = P.counters.template as<int>();
    w.xnd = P.Xnd.p;
    w.status = status_.template as<int>();
    const int nd = (int)depthNodes_.size();
    {
        ProfScope ps(st, kProfGatherScatter);
        LaunchSweepPregather<R>(fr, P.arena.template At<int2>(cp.pre), cp.preN, B, k, io, st, tc_);
    }
    for (int d = nd - 1; d >= 0; --d) {
        ProfScope ps(st, kProfSolveGemm, cp.fFlops[d], cp.fBytes[d]);
        const SweepVariant& v = cp.F(d);
        const SweepTile* tl = P.arena.template At<SweepTile>(v.tiles);
        TuneMark();
        bool done = false;
        if constexpr (std::is_same<R, float>::value) {
            if (v.tc) {
                LaunchSweepForwardTc(fr, tl, v.n, k, v.cols, w, st);
                done = true;
            }
        }
        if (!done) LaunchSweepForward<R>(fr, tl, v.n, v.chunk, k, w, st);
        TuneMark();
    }
    for (int d = 0; d < nd; ++d) {
        {
            ProfScope ps(st, kProfGatherScatter);
            LaunchSweepBackwardGather<R>(fr, P.arena.template At<int2>(cp.bGather[d]), cp.bGatherN[d], k, w, st,
                                         cp.B(d).tc);
        }
        ProfScope ps(st, kProfSolveGemm, cp.bFlops[d], cp.bBytes[d]);
        const SweepVariant& v = cp.B(d);
        const SweepTile* tl = P.arena.template At<SweepTile>(v.tiles);
        TuneMark();
        bool done = false;
        if constexpr (std::is_same<R, float>::value) {
            if (v.tc) {
                LaunchSweepBackwardTc(fr, tl, v.n, B, k, v.cols, io, w, st);
                done = true;
            }
        }
        if (!done) LaunchSweepBackward<R>(fr, tl, v.n, v.chunk, B, k, io, w, st);
        TuneMark();
    }
}

template <typename R>
void FactorStore<R>::SweepEager(z64* B, int ldk, int k) {
    const int np = an_.geom.numPanels;
    for (int i = 0; i < np - 1; ++i) SolvePanel(B, ldk, k, i, i == 0 ? 0 : 1, 0);
    SolvePanel(B, ldk, k, np - 1, np - 1 == 0 ? 0 : 1, 0);
    for (int i = np - 2; i >= 0; --i) SolvePanel(B, ldk, k, i, 2, 1);
}

template <typename R>
void FactorStore<R>::Sweep(z64* B, int ldk, int k, bool useGraph) {
    Profiler* prof = CurrentProfiler();
    const bool profiling = prof && prof->enabled;
    // recomputed panels factor inside the sweep (host-side slot tracking): eager
    if (!useGraph || profiling || !AllResident()) {
        ProfScope ps(h_.stream_, kProfSweep, SweepFlops(k), SweepBytes(k));
        SweepEager(B, ldk, k);
        return;
    }
    Plan(k);  // built outside the capture: it allocates and uploads
    for (const SweepGraph& g : graphs_)
        if (g.B == B && g.ldk == ldk && g.k == k) {
            CUDA_CHECK(cudaGraphLaunch(g.exec, h_.stream_));
            return;
        }
    if (graphs_.size() >= 8) {  // graphs of earlier work vectors (the scratch moved)
        CUDA_CHECK(cudaGraphExecDestroy(graphs_.front().exec));
        graphs_.erase(graphs_.begin());
    }
    cudaGraph_t graph;
    CUDA_CHECK(cudaStreamBeginCapture(h_.stream_, cudaStreamCaptureModeThreadLocal));
    SweepEager(B, ldk, k);
    CUDA_CHECK(cudaStreamEndCapture(h_.stream_, &graph));
    SweepGraph g{B, ldk, k, nullptr};
    CUDA_CHECK(cudaGraphInstantiate(&g.exec, graph, 0));
    CUDA_CHECK(cudaGraphDestroy(graph));
    graphs_.push_back(g);
    CUDA_CHECK(cudaGraphLaunch(g.exec, h_.stream_));
}

template <typename R>
double FactorStore<R>::PlanBytesPerRhs() const {
    double best = 0;
    for (int c = 0; c < 3; ++c) {
        if (!an_.classUsed[c]) continue;
        const ClassStructure& cs = an_.cls[c];
        double e = cs.nSub;
        for (size_t t = 0; t < cs.size.size(); ++t) e += 3.0 * (cs.size[t] + cs.usize[t]) + cs.size[t] + (cs.size[t] + cs.usize[t]);
        best = std::max(best, e);
    }
    return best * sizeof(cpx<R>);
}

template <typename R>
void FactorStore<R>::DropPlansExcept(int k) {
    for (size_t i = 0; i < graphs_.size();) {
        if (graphs_[i].k != k) {
            CUDA_CHECK(cudaGraphExecDestroy(graphs_[i].exec));
            graphs_.erase(graphs_.begin() + i);
        } else {
            ++i;
        }
    }
    for (size_t i = 0; i < plans_.size();) {
        if (plans_[i]->k != k) plans_.erase(plans_.begin() + i);
        else ++i;
    }
}

// Algorithmic work of one sweep: every panel but the top one is solved twice.
template <typename R>
double FactorStore<R>::SweepFlops(int k) const {
    const PanelGeometry& g = an_.geom;
    double f = 0;
    for (int p = 0; p < g.numPanels; ++p) {
        const ClassStructure& cs = an_.cls[g.Class(p)];
        double pf = 0;
        for (size_t t = 0; t < cs.size.size(); ++t) {
            const double s = cs.size[t], u = cs.usize[t];
            pf += 8.0 * k * 2 * ((s + u) * s - s * (s - 1) / 2);
        }
        f += (p == g.numPanels - 1 ? 1 : 2) * pf;
    }
    return f;
}

template <typename R>
double FactorStore<R>::SweepBytes(int k) const {
    const PanelGeometry& g = an_.geom;
    double b = 0;
    for (int p = 0; p < g.numPanels; ++p) {
        const ClassStructure& cs = an_.cls[g.Class(p)];
        double pb = 0;
        for (size_t t = 0; t < cs.size.size(); ++t) {
            const double s = cs.size[t], u = cs.usize[t];
            pb += 2.0 * sizeof(cpx<R>) * ((s + u) * s - s * (s - 1) / 2);
        }
        pb += 2.0 * 16.0 * k * g.Depth(p) * an_.disc.nx * an_.disc.ny;  // natural-order RHS in and out
        b += (p == g.numPanels - 1 ? 1 : 2) * pb;
    }
    return b;
}

template class FactorStore<double>;
template class FactorStore<float>;

// =====================================================================
// Helmholtz
// =====================================================================

Helmholtz::Helmholtz(const DiscParams& d, double damping, int planesPerPanel, int cutoff, int device)
    : damping_(damping), device_(device) {
    an_.Build(d, planesPerPanel, cutoff);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw PspError(kNoDevice, "no CUDA device");
    if (device < 0 || device >= count) throw PspError(kLogicError, "invalid CUDA device index");
    CUDA_CHECK(cudaSetDevice(device));
    CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    BuildTables();
}

Helmholtz::~Helmholtz() {
    cudaSetDevice(device_);
    f64_.reset();
    f32_.reset();
    if (stream_) cudaStreamDestroy(stream_);
}

void Helmholtz::BuildTables() {
    const DiscParams& d = an_.disc;
    const double hx = d.wx / (d.nx + 1), hy = d.wy / (d.ny + 1), hz = d.wz / (d.nz + 1);
    std::vector<Cd> t1, t2, t3;
    for (int i = -1; i <= d.nx; ++i)
        t1.push_back(Stretch(i, d.nx, d.bx, d.sigmax, hx, d.omega, d.frontBC == kPML, d.backBC == kPML, 0));
    for (int i = -1; i <= d.ny; ++i)
        t2.push_back(Stretch(i, d.ny, d.by, d.sigmay, hy, d.omega, d.leftBC == kPML, d.rightBC == kPML, 0));
    for (int i = -1; i <= d.nz; ++i)
        t3.push_back(Stretch(i, d.nz, d.bz, d.sigmaz, hz, d.omega, true, d.topBC == kPML, 0));
    std::vector<z64> v, iv;
    PushTable(v, iv, t1);
    v.insert(v.end(), iv.begin(), iv.end());
    UploadVector(dS1_, v, stream_);
    v.clear(); iv.clear();
    PushTable(v, iv, t2);
    v.insert(v.end(), iv.begin(), iv.end());
    UploadVector(dS2_, v, stream_);
    v.clear(); iv.clear();
    PushTable(v, iv, t3);
    v.insert(v.end(), iv.begin(), iv.end());
    UploadVector(dS3_, v, stream_);
    // artificial-PML tables of every panel subproblem (s3InvArtificial)
    const PanelGeometry& g = an_.geom;
    std::vector<Cd> ta;
    s3aOff_.assign(g.numPanels, 0);
    for (int p = 0; p < g.numPanels; ++p) {
        s3aOff_[p] = (int)ta.size();
        const int vSize = g.ClassVSize(g.Class(p)), vOff = g.SubVOffset(p);
        for (int i = -1; i <= vSize; ++i)
            ta.push_back(Stretch(vOff + i, d.nz, d.bz, d.sigmaz, hz, d.omega, true, d.topBC == kPML, vOff));
    }
    v.clear(); iv.clear();
    PushTable(v, iv, ta);
    const int na = (int)ta.size();
    v.insert(v.end(), iv.begin(), iv.end());
    UploadVector(dS3a_, v, stream_);

    sp_.nx = d.nx; sp_.ny = d.ny; sp_.nz = d.nz;
    sp_.ihx2 = 1.0 / (2 * hx * hx);
    sp_.ihy2 = 1.0 / (2 * hy * hy);
    sp_.ihz2 = 1.0 / (2 * hz * hz);
    sp_.omega = d.omega;
    sp_.s1 = dS1_.as<z64>(); sp_.is1 = sp_.s1 + (d.nx + 2);
    sp_.s2 = dS2_.as<z64>(); sp_.is2 = sp_.s2 + (d.ny + 2);
    sp_.s3 = dS3_.as<z64>(); sp_.is3 = sp_.s3 + (d.nz + 2);
    for (int c = 0; c < 3; ++c) {
        if (!an_.classUsed[c]) continue;
        const ClassStructure& cs = an_.cls[c];
        UploadVector(dNdToNat_[c], cs.ndToNat, stream_);
        UploadVector(dNbrRows_[c], cs.nbrRows, stream_);
        UploadVector(dRel_[c], cs.rel, stream_);
        UploadVector(dLower_[c], cs.lower, stream_);
        ap_.tabs.ndToNat[c] = dNdToNat_[c].as<int>();
        ap_.tabs.nbrRows[c] = dNbrRows_[c].as<int>();
    }
    ap_.sp = sp_;
    ap_.s3a = dS3a_.as<z64>();
    ap_.is3a = ap_.s3a + na;
    ap_.damping = damping_;
}

void Helmholtz::Initialize(const double* velocity, bool devicePtr, int panelScheme, int precision) {
    CUDA_CHECK(cudaSetDevice(device_));
    const auto t0 = std::chrono::steady_clock::now();
    if (an_.disc.omega == 0) throw PspError(kLogicError, "PML does not work at zero frequency");
    if (panelScheme < 0 || panelScheme > 1) throw PspError(kLogicError, "Invalid panelScheme value");
    if (precision < 0 || precision > 1) throw PspError(kLogicError, "Invalid precision mode");
    if (!velocity) throw PspError(kLogicError, "Velocity grid is incorrect");
    // A handle's discretization never changes, so a second Initialize at the
    // same precision keeps the factor store (storage, recorded factorization,
    // solve plans) and only refactors with the new velocity.
    const bool reuse = precision == precision_ && (precision == 0 ? (bool)f64_ : (bool)f32_);
    if (!reuse) Finalize();
    initialized_ = false;
    const int64_t N = NumUnknowns();
    if (!dVel_.p) dVel_.Allocate(N * sizeof(double));
    CUDA_CHECK(cudaMemcpyAsync(dVel_.p, velocity, N * sizeof(double),
                               devicePtr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream_));
    ap_.vel = dVel_.as<double>();
    precision_ = precision;
    ProfilerBinding bind(&prof_);
    if (precision == 0) {
        if (!f64_) f64_.reset(new FactorStore<double>(*this));
        f64_->Factor();
    } else {
        if (!f32_) f32_.reset(new FactorStore<float>(*this));
        f32_->Factor();
    }
    CUDA_CHECK(cudaStreamSynchronize(stream_));
    if (prof_.enabled) prof_.Flush();
    initialized_ = true;
    setupSeconds_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void Helmholtz::Finalize() {
    f64_.reset();
    f32_.reset();
    pool_.Release();
    initialized_ = false;
}

void* Helmholtz::Scratch(size_t bytes) {
    if (bytes > pool_.bytes) {
        pool_.Release();
        pool_.Allocate(bytes);
    }
    return pool_.p;
}

int Helmholtz::ResidentPanels() const {
    if (f64_) return f64_->ResidentPanels();
    if (f32_) return f32_->ResidentPanels();
    return 0;
}

int64_t Helmholtz::Refactorizations() const {
    if (f64_) return f64_->Refactorizations();
    if (f32_) return f32_->Refactorizations();
    return 0;
}

int64_t Helmholtz::factorBytes() const {
    if (f64_) return f64_->Bytes();
    if (f32_) return f32_->Bytes();
    return 0;
}

double Helmholtz::SweepFlops(int k) const {
    if (f64_) return f64_->SweepFlops(k);
    if (f32_) return f32_->SweepFlops(k);
    return 0;
}

double Helmholtz::SweepBytes(int k) const {
    if (f64_) return f64_->SweepBytes(k);
    if (f32_) return f32_->SweepBytes(k);
    return 0;
}

// Right-hand sides go through the sweep in blocks of equal width (at most
// kRhsBlock), so one solve plan serves every block.
constexpr int kRhsBlock = 64;
static int RhsBlockWidth(int k) {
    const int nb = (k + kRhsBlock - 1) / kRhsBlock;
    return (k + nb - 1) / nb;
}

void Helmholtz::Precondition(z64* B, int k, bool useGraph) {
    const int w = RhsBlockWidth(k);
    for (int r0 = 0; r0 < k; r0 += w) {
        const int kb = std::min(w, k - r0);
        if (f64_) f64_->Sweep(B + r0, k, kb, useGraph);
        else f32_->Sweep(B + r0, k, kb, useGraph);
    }
}

void Helmholtz::CheckSweepStatus() {
    const int st = f64_ ? f64_->ReadStatus() : (f32_ ? f32_->ReadStatus() : 0);
    if (st & 1) throw PspError(kRuntimeError, "zero or non-finite pivot in a recomputed panel factorization");
    if (st & 2) throw PspError(kRuntimeError, "a tensor-core pipeline wait timed out in the sweep");
}

void Helmholtz::PreconditionDevice(z64* B, int k) {
    if (!initialized_) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    CUDA_CHECK(cudaSetDevice(device_));
    ProfilerBinding bind(&prof_);
    Precondition(B, k, false);
    CUDA_CHECK(cudaStreamSynchronize(stream_));
    if (prof_.enabled) prof_.Flush();
    CheckSweepStatus();
}

void Helmholtz::SolvePanelDevice(z64* B, int k, int panel) {
    if (!initialized_) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    if (panel < 0 || panel >= an_.geom.numPanels) throw PspError(kLogicError, "panel index out of range");
    CUDA_CHECK(cudaSetDevice(device_));
    const int w = RhsBlockWidth(k);
    for (int r0 = 0; r0 < k; r0 += w) {
        const int kb = std::min(w, k - r0);
        if (f64_) f64_->SolvePanel(B + r0, k, kb, panel, 0, 0);
        else f32_->SolvePanel(B + r0, k, kb, panel, 0, 0);
    }
    CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void Helmholtz::SetPanelRange(int p0, int p1) {
    if (f64_ || f32_) throw PspError(kLogicError, "the panel range must be set before the first Initialize");
    if (p0 < 0 || p1 > an_.geom.numPanels || p0 >= p1) throw PspError(kLogicError, "invalid panel range");
    panelBegin_ = p0;
    panelEnd_ = p1;
}

void Helmholtz::SolvePanelSlab(z64* B, int k, int panel, int inMode, int outAccumulate, int zBase) {
    if (!initialized_) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    if (panel < 0 || panel >= an_.geom.numPanels) throw PspError(kLogicError, "panel index out of range");
    if (inMode < 0 || inMode > 2 || k < 1 || zBase < 0 || zBase >= an_.disc.nz)
        throw PspError(kLogicError, "invalid panel-solve arguments");
    // the lowest plane the panel solve touches: its top plane, or the plane
    // above it whose coupling in_mode 2 reads; in_mode 1 reads the plane
    // below its bottom one
    const PanelGeometry& g = an_.geom;
    const int zLow = an_.disc.nz - 1 - (g.LowV(panel) + g.Depth(panel) - 1) - (inMode == 2 ? 1 : 0);
    if (zLow < 0 || (inMode == 1 && g.LowV(panel) == 0))
        throw PspError(kLogicError, "panel " + std::to_string(panel) + " has no neighbouring panel for in_mode " +
                                        std::to_string(inMode));
    if (zBase > zLow)
        throw PspError(kLogicError, "the slab starts at plane " + std::to_string(zBase) + ", above plane " +
                                        std::to_string(zLow) + " that panel " + std::to_string(panel) + " needs");
    CUDA_CHECK(cudaSetDevice(device_));
    ProfilerBinding bind(&prof_);
    const int w = RhsBlockWidth(k);
    for (int r0 = 0; r0 < k; r0 += w) {
        const int kb = std::min(w, k - r0);
        if (f64_) f64_->SolvePanel(B + r0, k, kb, panel, inMode, outAccumulate, zBase);
        else f32_->SolvePanel(B + r0, k, kb, panel, inMode, outAccumulate, zBase);
    }
    CUDA_CHECK(cudaStreamSynchronize(stream_));
    CheckSweepStatus();
}

void Helmholtz::MultiplySlab(const z64* X, z64* Y, const z64* Bv, int k, int zFirst, int zCount, int zSlab) {
    if (!dVel_.p) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    // the slab must begin at or below the halo plane zFirst - 1 (which the
    // stencil of plane zFirst reads when it exists)
    if (k < 1 || zCount < 1 || zFirst < 0 || zFirst + zCount > an_.disc.nz || zSlab < 0 ||
        zSlab > std::max(0, zFirst - 1))
        throw PspError(kLogicError, "invalid slab multiply arguments");
    CUDA_CHECK(cudaSetDevice(device_));
    LaunchHelmholtzApplyPlanes(X, Y, Bv, dVel_.as<double>(), sp_, k, zFirst, zCount, zSlab, stream_);
    CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void Helmholtz::MultiplyDevice(z64* B, int k) {
    if (!dVel_.p) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    CUDA_CHECK(cudaSetDevice(device_));
    const int64_t nk = NumUnknowns() * k;
    DeviceBuffer tmp;
    tmp.Allocate(nk * sizeof(z64));
    LaunchHelmholtzApply(B, tmp.as<z64>(), nullptr, dVel_.as<double>(), sp_, k, stream_);
    CUDA_CHECK(cudaMemcpyAsync(B, tmp.p, nk * sizeof(z64), cudaMemcpyDeviceToDevice, stream_));
    CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void Helmholtz::GradientDevice(const z64* U, const z64* Z, int k, double* grad, bool accumulate) {
    if (!dVel_.p) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    if (k <= 0) throw PspError(kLogicError, "number of right-hand sides must be positive");
    CUDA_CHECK(cudaSetDevice(device_));
    LaunchVelocityGradient(U, Z, dVel_.as<double>(), sp_, k, grad, accumulate ? 1 : 0, stream_);
    CUDA_CHECK(cudaStreamSynchronize(stream_));
}

void Helmholtz::EnsureWorkspace(int k, int m, bool withCols) {
    const size_t nk = (size_t)NumUnknowns() * k;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t vec = al(nk * sizeof(z64));
    const size_t partial = al((size_t)ReduceBlocks(NumUnknowns(), k) * k * sizeof(z64));
    const size_t scal = al((size_t)(2 * k) * sizeof(double) + (size_t)(m + 1) * k * sizeof(z64));
    const size_t ybytes = al((size_t)m * k * sizeof(z64));
    const size_t total = vec * (4 + m + (withCols ? 1 : 0)) + partial + scal + ybytes;
    unsigned char* p = static_cast<unsigned char*>(Scratch(total));
    auto take = [&](size_t b) { unsigned char* q = p; p += b; return q; };
    wsCols_ = withCols ? reinterpret_cast<z64*>(take(vec)) : nullptr;
    wsX_ = reinterpret_cast<z64*>(take(vec));
    wsX0_ = reinterpret_cast<z64*>(take(vec));
    wsW_ = reinterpret_cast<z64*>(take(vec));
    wsB_ = reinterpret_cast<z64*>(take(vec));
    wsV_ = reinterpret_cast<z64*>(take(vec * m));
    wsPartial_ = take(partial);
    wsScal_ = take(scal);
    wsY_ = reinterpret_cast<z64*>(take(ybytes));
}

namespace {

// lapack::ComputeGivens semantics (solve.hpp:486-487):
// [c s; -conj(s) c] [f; g] = [rho; 0] with c real.
void Givens(Cd f, Cd g, double& c, Cd& s, Cd& rho) {
    const double af = std::abs(f), ag = std::abs(g);
    if (ag == 0) { c = 1; s = 0; rho = f; return; }
    if (af == 0) { c = 0; s = std::conj(g) / ag; rho = ag; return; }
    const double nrm = std::hypot(af, ag);
    c = af / nrm;
    s = (f / af) * std::conj(g) / nrm;
    rho = (f / af) * nrm;
}

bool AnyNaN(const std::vector<double>& v) {
    for (double x : v)
        if (x != x) return true;
    return false;
}

}  // namespace

double Helmholtz::GmresBytesPerRhs(int m) const {
    // V (m vectors), x, x0, w, b and a block's copy of its columns, the
    // solve plan's work vectors and the sweep autotuner's scratch
    double plan = 0;
    if (f64_) plan = f64_->PlanBytesPerRhs();
    if (f32_) plan = f32_->PlanBytesPerRhs();
    return (double)NumUnknowns() * sizeof(z64) * (m + 6) + plan;
}

int ChooseBlockWidth(int k, double availBytes, double perRhsBytes, int cap) {
    if (k < 1 || perRhsBytes <= 0) throw PspError(kLogicError, "need k >= 1 and a positive workspace size");
    const double fitD = std::floor(0.95 * availBytes / perRhsBytes);
    if (fitD < 1)
        throw PspError(kOutOfMemory, "the GMRES workspace of one right-hand side (" +
                                         std::to_string(perRhsBytes / 1e9) + " GB) does not fit in the " +
                                         std::to_string(availBytes / 1e9) +
                                         " GB of device memory left beside the factors");
    int fit = (int)std::min<double>(fitD, k);
    if (cap > 0) fit = std::min(fit, cap);
    const int nb = (k + fit - 1) / fit;
    int kb = (k + nb - 1) / nb;
    // whole 16-column sweep tiles when that still fits
    if (kb > 16 && kb % 16) {
        const int up = (kb + 15) / 16 * 16;
        if (up <= fit && up < k) kb = up;
    }
    return std::max(1, kb);
}

int Helmholtz::GmresBlockWidth(int k, int m) {
    const long long cap = EnvInt("PSP_B200_MAX_RHS_BLOCK", 0);
    size_t freeB = 0, totalB = 0;
    CUDA_CHECK(cudaMemGetInfo(&freeB, &totalB));
    // the scratch is reused for the workspace; the plan of the current width
    // (when built) is already counted as used memory
    const double avail = (double)freeB + (double)pool_.bytes - 0.5e9;
    return ChooseBlockWidth(k, avail, GmresBytesPerRhs(m), cap > 0 ? (int)std::min<long long>(cap, k) : 0);
}

void Helmholtz::SolveDevice(z64* B, int k, int m, double relTol, SolveStats* stats) {
    if (!initialized_) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    if (k < 1) throw PspError(kLogicError, "need at least one right-hand side");
    if (m < 1) throw PspError(kLogicError, "GMRES restart length must be positive");
    CUDA_CHECK(cudaSetDevice(device_));
    const int kb = GmresBlockWidth(k, m);
    if (kb >= k) {
        EnsureWorkspace(k, m, false);
        SolveBlock(B, k, m, relTol, stats);
        return;
    }
    const auto tStart = std::chrono::steady_clock::now();
    SolveStats local;
    SolveStats& S = stats ? *stats : local;
    S = SolveStats();
    S.converged = 1;
    const int64_t N = NumUnknowns();
    // blocks of equal width kb (one solve plan); a short last block is
    // padded with copies of its last column, whose results are dropped
    if (f64_) f64_->DropPlansExcept(RhsBlockWidth(kb));
    if (f32_) f32_->DropPlansExcept(RhsBlockWidth(kb));
    EnsureWorkspace(kb, m, true);
    z64* cols = wsCols_;
    const std::string viewBase = viewIterates_;
    std::vector<std::vector<Cd>> ritzPerRhs;
    int ritzCount = 0;
    struct Restore {
        Helmholtz& h;
        std::string base;
        ~Restore() { h.viewIterates_ = base; h.ritzRhsOffset_ = 0; }
    } restore{*this, viewBase};
    for (int c0 = 0; c0 < k; c0 += kb) {
        const int w = std::min(kb, k - c0);
        // columns [c0, c0 + w) of the [N][k] grid as a contiguous [N][kb] grid
        CUDA_CHECK(cudaMemcpy2DAsync(cols, kb * sizeof(z64), B + c0, k * sizeof(z64), w * sizeof(z64), N,
                                     cudaMemcpyDeviceToDevice, stream_));
        for (int c = w; c < kb; ++c)
            CUDA_CHECK(cudaMemcpy2DAsync(cols + c, kb * sizeof(z64), B + c0 + w - 1, k * sizeof(z64), sizeof(z64), N,
                                         cudaMemcpyDeviceToDevice, stream_));
        if (!viewBase.empty()) viewIterates_ = viewBase + "_rhs" + std::to_string(c0);
        ritzRhsOffset_ = c0;
        SolveStats s;
        EnsureWorkspace(kb, m, true);
        SolveBlock(cols, kb, m, relTol, &s);
        CUDA_CHECK(cudaMemcpy2DAsync(B + c0, k * sizeof(z64), cols, kb * sizeof(z64), w * sizeof(z64), N,
                                     cudaMemcpyDeviceToDevice, stream_));
        S.iterations = std::max(S.iterations, s.iterations);
        S.converged = S.converged && s.converged;
        S.luckyBreakdown = S.luckyBreakdown || s.luckyBreakdown;
        S.finalMaxRelResid = std::max(S.finalMaxRelResid, s.finalMaxRelResid);
        S.precondSeconds += s.precondSeconds;
        S.matvecSeconds += s.matvecSeconds;
        S.arnoldiSeconds += s.arnoldiSeconds;
        S.numPreconditions += s.numPreconditions;
        if (S.history.size() < s.history.size()) S.history.resize(s.history.size(), 0.0);
        for (size_t i = 0; i < s.history.size(); ++i) S.history[i] = std::max(S.history[i], s.history[i]);
        if (ritzK_ > 0) {
            for (int r = 0; r < w; ++r)
                ritzPerRhs.emplace_back(ritz_.begin() + (size_t)r * ritzCount_,
                                        ritz_.begin() + (size_t)(r + 1) * ritzCount_);
            ritzCount = std::max(ritzCount, ritzCount_);
        }
    }
    CUDA_CHECK(cudaStreamSynchronize(stream_));
    ritz_.clear();
    ritzCount_ = ritzK_ = 0;
    if ((int)ritzPerRhs.size() == k) {
        const double nan = std::numeric_limits<double>::quiet_NaN();
        ritz_.assign((size_t)k * ritzCount, Cd(nan, nan));
        for (int r = 0; r < k; ++r) std::copy(ritzPerRhs[r].begin(), ritzPerRhs[r].end(), ritz_.begin() + (size_t)r * ritzCount);
        ritzCount_ = ritzCount;
        ritzK_ = k;
    }
    S.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tStart).count();
}

void Helmholtz::SolveBlock(z64* B, int k, int m, double relTol, SolveStats* stats) {
    if (!initialized_) throw PspError(kNotInitialized, "DistHelmholtz is not initialized");
    if (k < 1) throw PspError(kLogicError, "need at least one right-hand side");
    if (m < 1) throw PspError(kLogicError, "GMRES restart length must be positive");
    CUDA_CHECK(cudaSetDevice(device_));
    const auto tStart = std::chrono::steady_clock::now();
    SolveStats local;
    SolveStats& S = stats ? *stats : local;
    S = SolveStats();
    const int64_t N = NumUnknowns(), nk = N * k;
    cudaStream_t st = stream_;
    z64* x = wsX_;
    z64* x0 = wsX0_;
    z64* w = wsW_;
    z64* b = wsB_;
    z64* V = wsV_;
    double* dNorm = static_cast<double*>(wsScal_);
    double* dDelta = dNorm + k;
    z64* dH = reinterpret_cast<z64*>(dDelta + k);
    z64* dY = wsY_;
    double* partialR = static_cast<double*>(wsPartial_);
    z64* partialC = static_cast<z64*>(wsPartial_);
    const int nblk = ReduceBlocks(N, k);
    const double* vel = dVel_.as<double>();
    // per-kernel profiling (when on) of the GMRES vector kernels: algorithmic
    // bytes = the [N][k] vectors each launch reads and writes
    const double vb = 16.0 * (double)nk;
    auto norms = [&](const z64* v, double* out) {
        {
            ProfScope ps(st, kProfVector, 4.0 * nk, vb);
            LaunchNormsPartial(v, N, k, partialR, st);
        }
        LaunchSumPartialReal(partialR, nblk, k, out, 1, st);
    };
    auto fetch = [&](void* dst, const void* src, size_t bytes) {
        CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    };
    // Phase timing with events on the solve stream, resolved at the sync
    // points GMRES needs anyway; per-kernel profiling nests inside when on.
    ProfilerBinding bind(&prof_);
    Profiler phases;
    phases.enabled = true;
    const double swFlops = SweepFlops(k), swBytes = SweepBytes(k);
    auto timed = [&](int cat, double f, double by, auto&& fn) {
        phases.Begin(st);
        fn();
        phases.End(st, cat, f, by);
    };
    auto precond = [&] {
        timed(kProfSweep, swFlops, swBytes, [&] { Precondition(w, k, true); });
        S.numPreconditions++;
    };
    const double mvFlops = 56.0 * nk, mvBytes = (double)N * (32.0 * k + 8);

    CUDA_CHECK(cudaMemcpyAsync(b, B, nk * sizeof(z64), cudaMemcpyDeviceToDevice, st));
    CUDA_CHECK(cudaMemsetAsync(x, 0, nk * sizeof(z64), st));
    CUDA_CHECK(cudaMemcpyAsync(w, b, nk * sizeof(z64), cudaMemcpyDeviceToDevice, st));
    std::vector<double> origResid(k), beta(k), delta(k), resid(k);
    norms(w, dNorm);
    fetch(origResid.data(), dNorm, k * sizeof(double));
    CUDA_CHECK(cudaStreamSynchronize(st));
    if (AnyNaN(origResid)) throw PspError(kRuntimeError, "Original residual norms had a NaN");

    std::vector<Cd> H((size_t)k * m * m), z((size_t)k * (m + 1)), sn((size_t)k * m), y((size_t)m * k), hcol;
    std::vector<double> cs((size_t)k * m);
    // HListCopy of solve.hpp:257-261: the unrotated Hessenberg matrices of
    // the first restart cycle, one m x m column-major block per RHS.
    ritz_.clear();
    ritzCount_ = ritzK_ = 0;
    bool firstBatch = ritzMode_ > 0;
    std::vector<Cd> Hfirst(firstBatch ? (size_t)k * m * m : 0, Cd(0));
    auto ritzValues = [&](int count) {
        ritzCount_ = count;
        ritzK_ = k;
        ritz_.assign((size_t)k * count, Cd(0));
        for (int r = 0; r < k; ++r) {
            const std::vector<Cd> ev = HessenbergEigenvalues(count, &Hfirst[(size_t)r * m * m], m);
            std::copy(ev.begin(), ev.end(), ritz_.begin() + (size_t)r * count);
            if (ritzMode_ > 1) {
                std::cout << "Ritz values for " << ritzRhsOffset_ + r
                          << "'th right-hand side before first restart:\n";
                for (int q = 0; q < count; ++q) std::cout << ev[q] << " ";
                std::cout << std::endl;
            }
        }
    };
    // viewIterates (solve.hpp:579-585): the current iterate in the grid's
    // natural [N][k] layout, written with WriteVolume.
    std::vector<z64> xHost;
    auto writeIterate = [&](int step) {
        xHost.resize(nk);
        CUDA_CHECK(cudaMemcpyAsync(xHost.data(), x, nk * sizeof(z64), cudaMemcpyDeviceToHost, st));
        CUDA_CHECK(cudaStreamSynchronize(st));
        GridWriteVolume(reinterpret_cast<const double*>(xHost.data()), an_.disc.nx, an_.disc.ny, an_.disc.nz, k,
                        true, viewIterates_ + "-" + std::to_string(step));
    };
    int it = 0;
    bool converged = false;
    double maxRel = 0;
    while (!converged) {
        CUDA_CHECK(cudaMemcpyAsync(x0, x, nk * sizeof(z64), cudaMemcpyDeviceToDevice, st));
        precond();
        norms(w, dNorm);
        fetch(beta.data(), dNorm, k * sizeof(double));
        CUDA_CHECK(cudaStreamSynchronize(st));
        if (AnyNaN(beta)) throw PspError(kRuntimeError, "beta list had a NaN");
        {
            ProfScope ps(st, kProfVector, 2.0 * nk, 2 * vb);
            LaunchScaleColumns(w, dNorm, V, N, k, st);
        }
        std::fill(z.begin(), z.end(), Cd(0));
        for (int r = 0; r < k; ++r) z[(size_t)r * (m + 1)] = beta[r];
        for (int j = 0; j < m; ++j) {
            timed(kProfStencil, mvFlops, mvBytes, [&] {
                ProfScope ps(st, kProfStencil, mvFlops, mvBytes);
                LaunchHelmholtzApply(V + (size_t)j * nk, w, nullptr, vel, sp_, k, st);
            });
            precond();
            phases.Begin(st);
            for (int i = 0; i <= j; ++i) {
                {
                    ProfScope ps(st, kProfVector, (i > 0 ? 16.0 : 8.0) * nk, (i > 0 ? 4 : 2) * vb);
                    LaunchMgsStep(w, i > 0 ? V + (size_t)(i - 1) * nk : nullptr,
                                  i > 0 ? dH + (size_t)(i - 1) * k : nullptr, V + (size_t)i * nk, N, k, partialC, st);
                }
                LaunchSumPartialComplex(partialC, nblk, k, dH + (size_t)i * k, st);
            }
            {
                ProfScope ps(st, kProfVector, 8.0 * nk, 3 * vb);
                LaunchAxpyColumns(w, V + (size_t)j * nk, dH + (size_t)j * k, N, k, st);
            }
            norms(w, dDelta);
            phases.End(st, kProfVector, 8.0 * 2 * (j + 1) * nk, 16.0 * (3 * (j + 1) + 2) * nk);
            hcol.resize((size_t)(j + 1) * k);
            fetch(hcol.data(), dH, (size_t)(j + 1) * k * sizeof(z64));
            fetch(delta.data(), dDelta, k * sizeof(double));
            CUDA_CHECK(cudaStreamSynchronize(st));
            if (AnyNaN(delta)) throw PspError(kRuntimeError, "delta list had a NaN");
            bool zeroDelta = false;
            for (double dv : delta) zeroDelta |= (dv == 0);
            if (zeroDelta) {
                // solve.hpp:405-414: the reference returns here without copying
                // the iterate back, so B keeps the right-hand sides.
                S.luckyBreakdown = 1;
                S.iterations = it;
                S.finalMaxRelResid = maxRel;
                S.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tStart).count();
                return;
            }
            if (firstBatch)
                for (int r = 0; r < k; ++r) {
                    Cd* Hr = &Hfirst[(size_t)r * m * m];
                    for (int i = 0; i <= j; ++i) Hr[(size_t)j * m + i] = Cd(hcol[(size_t)i * k + r]);
                    if (j + 1 != m) Hr[(size_t)j * m + j + 1] = delta[r];
                }
            phases.Begin(st);
            if (j + 1 != m) {
                ProfScope ps(st, kProfVector, 2.0 * nk, 2 * vb);
                LaunchScaleColumns(w, dDelta, V + (size_t)(j + 1) * nk, N, k, st);
            }
            for (int r = 0; r < k; ++r) {
                Cd* Hr = &H[(size_t)r * m * m];
                for (int i = 0; i <= j; ++i) Hr[(size_t)j * m + i] = Cd(hcol[(size_t)i * k + r]);
                for (int i = 0; i < j; ++i) {
                    const double c = cs[(size_t)r * m + i];
                    const Cd s = sn[(size_t)r * m + i];
                    const Cd a = Hr[(size_t)j * m + i], bb = Hr[(size_t)j * m + i + 1];
                    Hr[(size_t)j * m + i] = c * a + s * bb;
                    Hr[(size_t)j * m + i + 1] = -std::conj(s) * a + c * bb;
                }
                const Cd etajj = Hr[(size_t)j * m + j];
                if (etajj != etajj) throw PspError(kRuntimeError, "H(j,j) was NaN");
                double c;
                Cd s, rho;
                Givens(etajj, Cd(delta[r]), c, s, rho);
                if (c != c || s != s || rho != rho) throw PspError(kRuntimeError, "Givens rotation had a NaN");
                Hr[(size_t)j * m + j] = rho;
                cs[(size_t)r * m + j] = c;
                sn[(size_t)r * m + j] = s;
                Cd* zr = &z[(size_t)r * (m + 1)];
                const Cd zj = zr[j], zj1 = zr[j + 1];
                zr[j] = c * zj + s * zj1;
                zr[j + 1] = -std::conj(s) * zj + c * zj1;
                for (int i = j; i >= 0; --i) {
                    Cd acc = zr[i];
                    for (int q = i + 1; q <= j; ++q) acc -= Hr[(size_t)q * m + i] * y[(size_t)q * k + r];
                    y[(size_t)i * k + r] = acc / Hr[(size_t)i * m + i];
                }
            }
            CUDA_CHECK(cudaMemcpyAsync(dY, y.data(), (size_t)(j + 1) * k * sizeof(z64), cudaMemcpyHostToDevice, st));
            {
                ProfScope ps(st, kProfVector, 8.0 * (j + 1) * nk, (j + 3) * vb);
                LaunchCombine(x0, V, nk, dY, j + 1, x, N, k, st);
            }
            phases.End(st, kProfVector, 8.0 * (j + 1) * nk, 16.0 * (j + 3) * nk);
            timed(kProfStencil, mvFlops, mvBytes + 16.0 * nk, [&] {
                ProfScope ps(st, kProfStencil, mvFlops, mvBytes + 16.0 * nk);
                LaunchHelmholtzApply(x, w, b, vel, sp_, k, st);
            });
            norms(w, dNorm);
            fetch(resid.data(), dNorm, k * sizeof(double));
            CUDA_CHECK(cudaStreamSynchronize(st));
            phases.Flush();
            if (AnyNaN(resid)) throw PspError(kRuntimeError, "resid norm list has NaN");
            maxRel = 0;
            for (int r = 0; r < k; ++r) maxRel = std::max(maxRel, resid[r] / origResid[r]);
            S.history.push_back(maxRel);
            if (maxRel < relTol) {
                converged = true;
                ++it;
                break;
            }
            if (!viewIterates_.empty()) writeIterate(it);
            ++it;
            if (maxIterations_ > 0 && it >= maxIterations_) break;
        }
        // solve.hpp:589-608: after the first restart cycle, `it` is its
        // number of inner steps.
        if (firstBatch) ritzValues(it);
        firstBatch = false;
        if (maxIterations_ > 0 && it >= maxIterations_) break;
    }
    CUDA_CHECK(cudaMemcpyAsync(B, x, nk * sizeof(z64), cudaMemcpyDeviceToDevice, st));
    CUDA_CHECK(cudaStreamSynchronize(st));
    phases.Flush();
    if (prof_.enabled) prof_.Flush();
    CheckSweepStatus();
    S.precondSeconds = phases.totals[kProfSweep].ms * 1e-3;
    S.matvecSeconds = phases.totals[kProfStencil].ms * 1e-3;
    S.arnoldiSeconds = phases.totals[kProfVector].ms * 1e-3;
    S.iterations = it;
    S.converged = converged ? 1 : 0;
    S.finalMaxRelResid = maxRel;
    S.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tStart).count();
}

}  // namespace psp_b200
