// C ABI over psp_b200::Helmholtz: converts exceptions into status codes.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/psp_b200.h"
#include "grid_io.hpp"
#include "handle.hpp"
#include "ritz.hpp"
#include "solver.hpp"

using psp_b200::Helmholtz;
using psp_b200::PspError;

namespace {

thread_local std::string g_lastError;

template <typename F>
int Guard(F&& fn) {
    try {
        fn();
        g_lastError.clear();
        return PSP_CU_OK;
    } catch (const PspError& e) {
        g_lastError = e.what();
        return e.code;
    } catch (const std::bad_alloc& e) {
        g_lastError = "host allocation failed";
        return PSP_CU_OUT_OF_MEMORY;
    } catch (const std::logic_error& e) {
        g_lastError = e.what();
        return PSP_CU_LOGIC_ERROR;
    } catch (const std::exception& e) {
        g_lastError = e.what();
        return PSP_CU_RUNTIME_ERROR;
    }
}

int CheckHandle(const psp_cu_handle* h) {
    if (!h || !h->solver) {
        g_lastError = "null handle";
        return PSP_CU_LOGIC_ERROR;
    }
    return PSP_CU_OK;
}

void FillStats(const psp_b200::SolveStats& s, psp_cu_stats* out) {
    if (!out) return;
    out->iterations = s.iterations;
    out->converged = s.converged;
    out->lucky_breakdown = s.luckyBreakdown;
    out->final_max_rel_resid = s.finalMaxRelResid;
    out->solve_seconds = s.seconds;
    out->precondition_seconds = s.precondSeconds;
    out->matvec_seconds = s.matvecSeconds;
    out->arnoldi_seconds = s.arnoldiSeconds;
    out->num_preconditions = s.numPreconditions;
}

// Runs fn on a device copy of the host grid B and copies the result back,
// through the handle's pinned staging and device scratch.
template <typename F>
void OnDeviceCopy(psp_cu_handle* h, double* B, int k, F&& fn) {
    if (!B) throw PspError(PSP_CU_LOGIC_ERROR, "null grid");
    if (k < 1) throw PspError(PSP_CU_LOGIC_ERROR, "need at least one right-hand side");
    Helmholtz* s = h->solver;
    CUDA_CHECK(cudaSetDevice(s->device()));
    const size_t bytes = (size_t)s->NumUnknowns() * k * 2 * sizeof(double);
    void* d = h->io.Device(bytes);
    h->io.ToDevice(d, B, bytes, s->stream());
    fn(static_cast<psp_b200::z64*>(d));
    h->io.ToHost(B, d, bytes, s->stream());
}

// A device grid argument: a pointer and at least one right-hand side.
void CheckDeviceGrid(const void* d, int k) {
    if (!d) throw PspError(PSP_CU_LOGIC_ERROR, "null grid");
    if (k < 1) throw PspError(PSP_CU_LOGIC_ERROR, "need at least one right-hand side");
}

}  // namespace

namespace psp_b200 {
void SetLastError(const std::string& msg) { g_lastError = msg; }
}  // namespace psp_b200

extern "C" {

const char* psp_cu_last_error(void) { return g_lastError.c_str(); }

int psp_cu_create(const psp_cu_disc* disc, double damping, int planes_per_panel, int cutoff, int device,
                  psp_cu_handle** out) {
    if (!disc || !out) {
        g_lastError = "null argument";
        return PSP_CU_LOGIC_ERROR;
    }
    *out = nullptr;
    return Guard([&] {
        psp_b200::DiscParams d;
        static_assert(sizeof(psp_b200::DiscParams) == sizeof(psp_cu_disc), "disc layout");
        std::memcpy(&d, disc, sizeof(d));
        Helmholtz* s = new Helmholtz(d, damping, planes_per_panel, cutoff, device);
        *out = new psp_cu_handle{s};
    });
}

void psp_cu_destroy(psp_cu_handle* h) {
    if (!h) return;
    delete h->solver;
    delete h;
}

int psp_cu_initialize(psp_cu_handle* h, const double* velocity, int panel_scheme, int precision) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        // argument errors are reported by Initialize itself, in its order
        if (!velocity) return h->solver->Initialize(nullptr, false, panel_scheme, precision);
        CUDA_CHECK(cudaSetDevice(h->solver->device()));
        const size_t bytes = (size_t)h->solver->NumUnknowns() * sizeof(double);
        void* d = h->io.Device(bytes);
        h->io.ToDevice(d, velocity, bytes, h->solver->stream());
        h->solver->Initialize(static_cast<const double*>(d), true, panel_scheme, precision);
    });
}

int psp_cu_initialize_device(psp_cu_handle* h, const double* d_velocity, int panel_scheme, int precision) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] { h->solver->Initialize(d_velocity, true, panel_scheme, precision); });
}

int psp_cu_initialize_batch(psp_cu_handle* const* h, const double* const* velocity, int count, int panel_scheme,
                            int precision, int* failed) {
    if (failed) *failed = -1;
    if (count < 0 || (count > 0 && (!h || !velocity))) {
        psp_b200::SetLastError("invalid batch");
        return PSP_CU_LOGIC_ERROR;
    }
    for (int i = 0; i < count; ++i) {
        if (int e = psp_cu_initialize(h[i], velocity[i], panel_scheme, precision)) {
            if (failed) *failed = i;
            return e;
        }
    }
    return PSP_CU_OK;
}

int psp_cu_solve_batch(psp_cu_handle* const* h, double* const* B, const int* k, int count, int m, double rel_tol,
                       psp_cu_stats* stats, int* failed) {
    if (failed) *failed = -1;
    if (count < 0 || (count > 0 && (!h || !B || !k))) {
        psp_b200::SetLastError("invalid batch");
        return PSP_CU_LOGIC_ERROR;
    }
    for (int i = 0; i < count; ++i) {
        if (int e = psp_cu_solve(h[i], B[i], k[i], m, rel_tol, stats ? stats + i : nullptr)) {
            if (failed) *failed = i;
            return e;
        }
    }
    return PSP_CU_OK;
}

int psp_cu_solve(psp_cu_handle* h, double* B, int k, int m, double rel_tol, psp_cu_stats* stats) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        if (!h->solver->Initialized()) throw PspError(PSP_CU_NOT_INITIALIZED, "DistHelmholtz is not initialized");
        psp_b200::SolveStats s;
        OnDeviceCopy(h, B, k, [&](psp_b200::z64* d) { h->solver->SolveDevice(d, k, m, rel_tol, &s); });
        FillStats(s, stats);
    });
}

int psp_cu_solve_device(psp_cu_handle* h, double* d_B, int k, int m, double rel_tol, psp_cu_stats* stats) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        CheckDeviceGrid(d_B, k);
        psp_b200::SolveStats s;
        h->solver->SolveDevice(reinterpret_cast<psp_b200::z64*>(d_B), k, m, rel_tol, &s);
        FillStats(s, stats);
    });
}

int psp_cu_finalize(psp_cu_handle* h) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] { h->solver->Finalize(); });
}

int psp_cu_multiply(psp_cu_handle* h, double* B, int k) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        OnDeviceCopy(h, B, k, [&](psp_b200::z64* d) { h->solver->MultiplyDevice(d, k); });
    });
}

int psp_cu_precondition(psp_cu_handle* h, double* B, int k) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        if (!h->solver->Initialized()) throw PspError(PSP_CU_NOT_INITIALIZED, "DistHelmholtz is not initialized");
        OnDeviceCopy(h, B, k, [&](psp_b200::z64* d) { h->solver->PreconditionDevice(d, k); });
    });
}

int psp_cu_multiply_device(psp_cu_handle* h, double* d_B, int k) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        CheckDeviceGrid(d_B, k);
        h->solver->MultiplyDevice(reinterpret_cast<psp_b200::z64*>(d_B), k);
    });
}

int psp_cu_precondition_device(psp_cu_handle* h, double* d_B, int k) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        CheckDeviceGrid(d_B, k);
        h->solver->PreconditionDevice(reinterpret_cast<psp_b200::z64*>(d_B), k);
    });
}

int psp_cu_gradient_device(psp_cu_handle* h, const double* d_U, const double* d_Z, int k, double* d_grad,
                           int accumulate) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        if (!d_U || !d_Z || !d_grad) throw PspError(PSP_CU_LOGIC_ERROR, "null grid");
        h->solver->GradientDevice(reinterpret_cast<const psp_b200::z64*>(d_U),
                                  reinterpret_cast<const psp_b200::z64*>(d_Z), k, d_grad, accumulate != 0);
    });
}

int psp_cu_solve_panel(psp_cu_handle* h, double* B, int k, int panel) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        if (!h->solver->Initialized()) throw PspError(PSP_CU_NOT_INITIALIZED, "DistHelmholtz is not initialized");
        OnDeviceCopy(h, B, k, [&](psp_b200::z64* d) { h->solver->SolvePanelDevice(d, k, panel); });
    });
}

int psp_cu_set_panel_range(psp_cu_handle* h, int p0, int p1) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] { h->solver->SetPanelRange(p0, p1); });
}

int psp_cu_solve_panel_slab(psp_cu_handle* h, double* d_B, int k, int panel, int in_mode, int out_accumulate,
                            int z_base) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        if (!d_B) throw PspError(PSP_CU_LOGIC_ERROR, "null grid");
        h->solver->SolvePanelSlab(reinterpret_cast<psp_b200::z64*>(d_B), k, panel, in_mode, out_accumulate, z_base);
    });
}

int psp_cu_multiply_slab(psp_cu_handle* h, const double* d_X, double* d_Y, const double* d_Bv, int k, int z_first,
                         int z_count, int z_slab) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        if (!d_X || !d_Y) throw PspError(PSP_CU_LOGIC_ERROR, "null grid");
        h->solver->MultiplySlab(reinterpret_cast<const psp_b200::z64*>(d_X), reinterpret_cast<psp_b200::z64*>(d_Y),
                                reinterpret_cast<const psp_b200::z64*>(d_Bv), k, z_first, z_count, z_slab);
    });
}

int psp_cu_set_max_iterations(psp_cu_handle* h, int max_iterations) {
    if (int e = CheckHandle(h)) return e;
    h->solver->SetMaxIterations(max_iterations);
    return PSP_CU_OK;
}

int psp_cu_set_view_iterates(psp_cu_handle* h, const char* basename) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] { h->solver->SetViewIterates(basename ? std::string(basename) : std::string()); });
}

int psp_cu_set_ritz_values(psp_cu_handle* h, int mode) {
    if (int e = CheckHandle(h)) return e;
    if (mode < 0 || mode > 2) {
        g_lastError = "Ritz value mode must be 0, 1 or 2";
        return PSP_CU_LOGIC_ERROR;
    }
    h->solver->SetRitzValues(mode);
    return PSP_CU_OK;
}

int psp_cu_get_ritz_values(const psp_cu_handle* h, int* count, int* num_rhs, double* out) {
    if (int e = CheckHandle(h)) return e;
    const Helmholtz& s = *h->solver;
    if (count) *count = s.ritzCount();
    if (num_rhs) *num_rhs = s.ritzNumRhs();
    if (out && !s.ritzValues().empty())
        std::memcpy(out, s.ritzValues().data(), s.ritzValues().size() * sizeof(std::complex<double>));
    return PSP_CU_OK;
}

int psp_cu_hessenberg_eigenvalues(int n, const double* H, int ldh, double* w) {
    return Guard([&] {
        if (n > 0 && !w) throw std::logic_error("eigenvalue output is null");
        const auto ev = psp_b200::HessenbergEigenvalues(n, reinterpret_cast<const std::complex<double>*>(H), ldh);
        if (n > 0) std::memcpy(w, ev.data(), ev.size() * sizeof(std::complex<double>));
    });
}

int psp_cu_geometry(const psp_cu_handle* h, int* num_panels, int* info) {
    if (int e = CheckHandle(h)) return e;
    const psp_b200::PanelGeometry& g = h->solver->analysis().geom;
    if (num_panels) *num_panels = g.numPanels;
    if (info)
        for (int p = 0; p < g.numPanels; ++p) {
            info[4 * p + 0] = g.LowV(p);
            info[4 * p + 1] = g.Depth(p);
            info[4 * p + 2] = g.Padding(p);
            info[4 * p + 3] = g.Class(p);
        }
    return PSP_CU_OK;
}

int psp_cu_panel_geometry(const psp_cu_disc* disc, int planes_per_panel, int* num_panels, int* info) {
    if (!disc) {
        g_lastError = "null argument";
        return PSP_CU_LOGIC_ERROR;
    }
    return Guard([&] {
        psp_b200::DiscParams d;
        std::memcpy(&d, disc, sizeof(d));
        psp_b200::PanelGeometry g;
        g.Init(d, planes_per_panel);
        if (num_panels) *num_panels = g.numPanels;
        if (info)
            for (int p = 0; p < g.numPanels; ++p) {
                info[4 * p + 0] = g.LowV(p);
                info[4 * p + 1] = g.Depth(p);
                info[4 * p + 2] = g.Padding(p);
                info[4 * p + 3] = g.Class(p);
            }
    });
}

int psp_cu_get_stream(const psp_cu_handle* h, void** stream) {
    if (int e = CheckHandle(h)) return e;
    if (stream) *stream = (void*)h->solver->stream();
    return PSP_CU_OK;
}

int psp_cu_set_profiling(psp_cu_handle* h, int on) {
    if (int e = CheckHandle(h)) return e;
    h->solver->profiler().enabled = on != 0;
    return PSP_CU_OK;
}

int psp_cu_profile_reset(psp_cu_handle* h) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] { h->solver->profiler().Reset(); });
}

int psp_cu_profile_get(psp_cu_handle* h, int category, long long* launches, double* ms, double* flops,
                       double* bytes) {
    if (int e = CheckHandle(h)) return e;
    if (category < 0 || category >= psp_b200::kProfNumCategories) {
        g_lastError = "profile category out of range";
        return PSP_CU_LOGIC_ERROR;
    }
    return Guard([&] {
        psp_b200::Profiler& p = h->solver->profiler();
        p.Flush();
        const psp_b200::ProfileTotals& t = p.totals[category];
        if (launches) *launches = t.launches;
        if (ms) *ms = t.ms;
        if (flops) *flops = t.flops;
        if (bytes) *bytes = t.bytes;
    });
}

int psp_cu_sweep_cost(const psp_cu_handle* h, int k, double* flops, double* bytes) {
    if (int e = CheckHandle(h)) return e;
    if (flops) *flops = h->solver->SweepFlops(k);
    if (bytes) *bytes = h->solver->SweepBytes(k);
    return PSP_CU_OK;
}

int psp_cu_analyze_class(const psp_cu_disc* disc, int planes_per_panel, int cutoff, int cls, int* num_nodes,
                         int* vsize, int* info, int* nd_to_nat) {
    if (!disc) {
        g_lastError = "null argument";
        return PSP_CU_LOGIC_ERROR;
    }
    return Guard([&] {
        psp_b200::DiscParams d;
        std::memcpy(&d, disc, sizeof(d));
        psp_b200::Analysis an;
        an.Build(d, planes_per_panel, cutoff);
        if (cls < 0 || cls > 2 || !an.classUsed[cls]) throw std::logic_error("panel class not present");
        const psp_b200::ClassStructure& cs = an.cls[cls];
        const int nn = (int)an.tree.nodes.size();
        if (num_nodes) *num_nodes = nn;
        if (vsize) *vsize = cs.vSize;
        if (info)
            for (int t = 0; t < nn; ++t) {
                info[4 * t + 0] = cs.off[t];
                info[4 * t + 1] = cs.size[t];
                info[4 * t + 2] = cs.usize[t];
                info[4 * t + 3] = an.tree.nodes[t].parent;
            }
        if (nd_to_nat) std::memcpy(nd_to_nat, cs.ndToNat.data(), sizeof(int) * cs.ndToNat.size());
    });
}

int psp_cu_setup_info(const psp_cu_handle* h, double* setup_seconds, long long* factor_bytes) {
    if (int e = CheckHandle(h)) return e;
    if (setup_seconds) *setup_seconds = h->solver->setupSeconds();
    if (factor_bytes) *factor_bytes = (long long)h->solver->factorBytes();
    return PSP_CU_OK;
}

int psp_cu_memory_info(const psp_cu_handle* h, int* resident_panels, int* num_panels, long long* refactorizations,
                       long long* scratch_bytes) {
    if (int e = CheckHandle(h)) return e;
    if (resident_panels) *resident_panels = h->solver->ResidentPanels();
    if (num_panels) *num_panels = h->solver->analysis().geom.numPanels;
    if (refactorizations) *refactorizations = (long long)h->solver->Refactorizations();
    if (scratch_bytes) *scratch_bytes = (long long)h->solver->ScratchBytes();
    return PSP_CU_OK;
}

int psp_cu_solve_block_width(psp_cu_handle* h, int k, int m, int* width) {
    if (int e = CheckHandle(h)) return e;
    return Guard([&] {
        if (!width) throw PspError(PSP_CU_LOGIC_ERROR, "null output");
        CUDA_CHECK(cudaSetDevice(h->solver->device()));
        *width = h->solver->SolveBlockWidth(k, m);
    });
}

int psp_cu_plan_block_width(int k, double avail_bytes, double per_rhs_bytes, int cap, int* width) {
    return Guard([&] {
        if (!width) throw PspError(PSP_CU_LOGIC_ERROR, "null output");
        *width = psp_b200::ChooseBlockWidth(k, avail_bytes, per_rhs_bytes, cap);
    });
}

int psp_cu_grid_load(const char* filename, int nx, int ny, int nz, int num_scalars, int is_complex, int order,
                     double* d_out) {
    return Guard([&] {
        if (!filename) throw PspError(PSP_CU_LOGIC_ERROR, "null file name");
        psp_b200::GridLoad(filename, nx, ny, nz, num_scalars * (is_complex ? 2 : 1), order, d_out);
    });
}

int psp_cu_grid_interpolate(const double* d_in, int nx_old, int ny_old, int nz_old, int num_scalars, int is_complex,
                            double* d_out, int nx, int ny, int nz) {
    return Guard([&] {
        psp_b200::GridInterpolate(d_in, nx_old, ny_old, nz_old, num_scalars * (is_complex ? 2 : 1), d_out, nx, ny,
                                  nz);
    });
}

int psp_cu_grid_write_plane(const double* data, int nx, int ny, int nz, int num_scalars, int is_complex,
                            int plane_type, int which_plane, const char* basename) {
    return Guard([&] {
        if (!basename) throw PspError(PSP_CU_LOGIC_ERROR, "null base name");
        psp_b200::GridWritePlane(data, nx, ny, nz, num_scalars, is_complex != 0, plane_type, which_plane, basename);
    });
}

int psp_cu_grid_write_volume(const double* data, int nx, int ny, int nz, int num_scalars, int is_complex,
                             const char* basename) {
    return Guard([&] {
        if (!basename) throw PspError(PSP_CU_LOGIC_ERROR, "null base name");
        psp_b200::GridWriteVolume(data, nx, ny, nz, num_scalars, is_complex != 0, basename);
    });
}

}  // extern "C"
