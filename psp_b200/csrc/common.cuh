// Shared device helpers: a complex POD type usable for float and double, and
// CUDA error plumbing that turns every failure into an exception carrying a
// psp status code (the C ABI converts it back into a return code).
#pragma once
#include <utility>
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace psp_b200 {

template <typename R>
struct alignas(2 * sizeof(R)) cpx {
    R re, im;
};

template <typename R>
__host__ __device__ __forceinline__ cpx<R> mk(R re, R im) {
    cpx<R> z;
    z.re = re;
    z.im = im;
    return z;
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator+(cpx<R> a, cpx<R> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator-(cpx<R> a, cpx<R> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator-(cpx<R> a) { return mk(-a.re, -a.im); }
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator*(cpx<R> a, cpx<R> b) {
    return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator*(R s, cpx<R> a) { return mk(s * a.re, s * a.im); }
template <typename R>
__host__ __device__ __forceinline__ cpx<R>& operator+=(cpx<R>& a, cpx<R> b) { a.re += b.re; a.im += b.im; return a; }
template <typename R>
__host__ __device__ __forceinline__ cpx<R>& operator-=(cpx<R>& a, cpx<R> b) { a.re -= b.re; a.im -= b.im; return a; }
// acc += a*b
template <typename R>
__host__ __device__ __forceinline__ void cfma(cpx<R>& acc, cpx<R> a, cpx<R> b) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(-a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(a.im, b.re, acc.im);
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> cinv(cpx<R> a) {
    const R d = a.re * a.re + a.im * a.im;
    return mk(a.re / d, -a.im / d);
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> cdiv(cpx<R> a, cpx<R> b) {
    const R d = b.re * b.re + b.im * b.im;
    return mk((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
template <typename R>
__host__ __device__ __forceinline__ R cabs2(cpx<R> a) { return a.re * a.re + a.im * a.im; }
template <typename To, typename From>
__host__ __device__ __forceinline__ cpx<To> ccast(cpx<From> a) { return mk((To)a.re, (To)a.im); }

typedef cpx<double> z64;   // complex double
typedef cpx<float> c32;    // complex single

// Status codes of the C ABI (include/psp_b200.h).
enum Status {
    kOk = 0,
    kLogicError = 1,      // std::logic_error in the reference (bad arguments, shallow domain, ...)
    kRuntimeError = 2,    // std::runtime_error in the reference (NaN in GMRES, ...)
    kCudaError = 3,
    kOutOfMemory = 4,
    kNotInitialized = 5,
    kNoDevice = 6,
};

struct PspError : std::runtime_error {
    int code;
    PspError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void CudaCheck(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? kOutOfMemory : kCudaError;
        throw PspError(code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
                                 std::to_string(line) + ")");
    }
}
#define CUDA_CHECK(x) ::psp_b200::CudaCheck((x), #x, __FILE__, __LINE__)
#define CUDA_LAUNCH_CHECK() ::psp_b200::CudaCheck(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

inline unsigned CeilDiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// Programmatic dependent launch.  A kernel launched with LaunchPdl may start
// while the kernel before it in the stream is still running: it calls
// PdlTrigger() so that the kernel after it may be scheduled likewise, and
// PdlWait() (which returns once the preceding kernel has completed and its
// memory is visible) before touching any data that kernel reads or writes.
// A dependent grid starts only after every block of its predecessor has
// triggered, so waiting blocks never hold back unscheduled ones.
__device__ __forceinline__ void PdlTrigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void PdlWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
void LaunchPdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CudaCheck(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...), "kernel launch", __FILE__, __LINE__);
}

}  // namespace psp_b200
