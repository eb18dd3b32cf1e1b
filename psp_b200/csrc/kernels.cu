// CUDA-core kernels of the solve: on-the-fly 7-point PML stencil, batched
// complex GEMM over task lists, frontal LDL^T building blocks, multifrontal
// gathers/scatters of the panel solves and the multi-RHS GMRES vector ops.
#include <algorithm>

#include "kernels.cuh"

namespace psp_b200 {

namespace {

constexpr int kThreads = 256;

// Face and centre terms of one stencil row (initialize_finalize.hpp:527-587
// and 589-651).  s3M and the three s3 reciprocals come from either the global
// or the panel's artificial table; omega is omega (+ i*damping for panels).
struct Terms {
    z64 c, xL, xR, yL, yR, vL, vR;
};

__device__ __forceinline__ Terms StencilAt(const StencilParams& sp, int x, int y, z64 s3M, z64 is3L, z64 is3M,
                                           z64 is3R, z64 omega, double alpha) {
    const z64 s1M = sp.s1[x + 1], s2M = sp.s2[y + 1];
    const z64 cx = s2M * s3M, cy = s1M * s3M, cz = s1M * s2M;
    Terms t;
    t.xL = sp.ihx2 * (cx * (sp.is1[x] + sp.is1[x + 1]));
    t.xR = sp.ihx2 * (cx * (sp.is1[x + 2] + sp.is1[x + 1]));
    t.yL = sp.ihy2 * (cy * (sp.is2[y] + sp.is2[y + 1]));
    t.yR = sp.ihy2 * (cy * (sp.is2[y + 2] + sp.is2[y + 1]));
    t.vL = sp.ihz2 * (cz * (is3L + is3M));
    t.vR = sp.ihz2 * (cz * (is3R + is3M));
    const z64 w = mk(omega.re / alpha, omega.im / alpha);
    t.c = (t.xL + t.xR + t.yL + t.yR + t.vL + t.vR) - (w * w) * (cz * s3M);
    return t;
}

// ---------------------------------------------------------------- stencil apply

constexpr int kApplyTX = 64;

__global__ void __launch_bounds__(kThreads) helmholtz_apply_kernel(const z64* __restrict__ x, z64* __restrict__ y,
                                                                   const z64* __restrict__ b,
                                                                   const double* __restrict__ vel, StencilParams sp,
                                                                   int k, int zFirst, int zSlab) {
    __shared__ z64 coef[kApplyTX][7];
    const int x0 = blockIdx.x * kApplyTX, yy = blockIdx.y, zz = zFirst + (int)blockIdx.z;
    const int nx = sp.nx, ny = sp.ny, nz = sp.nz;
    const int64_t nxy = (int64_t)nx * ny;
    const int npts = min(kApplyTX, nx - x0);
    const int v = nz - 1 - zz;
    if ((int)threadIdx.x < npts) {
        const int xx = x0 + threadIdx.x;
        const Terms t = StencilAt(sp, xx, yy, sp.s3[v + 1], sp.is3[v], sp.is3[v + 1], sp.is3[v + 2],
                                  mk(sp.omega, 0.0), vel[xx + yy * (int64_t)nx + zz * nxy]);
        coef[threadIdx.x][0] = t.c;
        coef[threadIdx.x][1] = -t.xL;
        coef[threadIdx.x][2] = -t.xR;
        coef[threadIdx.x][3] = -t.yL;
        coef[threadIdx.x][4] = -t.yR;
        coef[threadIdx.x][5] = -t.vL;
        coef[threadIdx.x][6] = -t.vR;
    }
    __syncthreads();
    const int64_t base = x0 + yy * (int64_t)nx + (zz - zSlab) * nxy;  // storage: planes from zSlab
    const int64_t sx = k, sy = (int64_t)nx * k, sz = nxy * k;
    for (int e = threadIdx.x; e < npts * k; e += blockDim.x) {
        const int p = e / k, r = e - p * k;
        const int xx = x0 + p;
        const int64_t idx = (base + p) * k + r;
        const z64* xp = x + idx;
        z64 acc = coef[p][0] * xp[0];
        if (xx > 0) cfma(acc, coef[p][1], xp[-sx]);
        if (xx + 1 < nx) cfma(acc, coef[p][2], xp[sx]);
        if (yy > 0) cfma(acc, coef[p][3], xp[-sy]);
        if (yy + 1 < ny) cfma(acc, coef[p][4], xp[sy]);
        if (zz + 1 < nz) cfma(acc, coef[p][5], xp[sz]);   // v-1 neighbour
        if (zz > 0) cfma(acc, coef[p][6], xp[-sz]);       // v+1 neighbour
        y[idx] = b ? b[idx] - acc : acc;
    }
}

// ---------------------------------------------------------------- velocity gradient

__global__ void __launch_bounds__(kThreads) velocity_gradient_kernel(const z64* __restrict__ U,
                                                                     const z64* __restrict__ Z,
                                                                     const double* __restrict__ vel, StencilParams sp,
                                                                     int k, double* __restrict__ grad, int accumulate) {
    const int64_t nxy = (int64_t)sp.nx * sp.ny, n = nxy * sp.nz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int xx = (int)(i % sp.nx), yy = (int)((i / sp.nx) % sp.ny), zz = (int)(i / nxy);
        const int v = sp.nz - 1 - zz;
        const double a = vel[i];
        const z64 s = sp.s1[xx + 1] * sp.s2[yy + 1] * sp.s3[v + 1];
        const z64 dA = (2.0 * sp.omega * sp.omega / (a * a * a)) * s;
        z64 acc = mk(0.0, 0.0);
        for (int r = 0; r < k; ++r) cfma(acc, Z[i * k + r], U[i * k + r]);
        const double g = -(dA * acc).re;
        grad[i] = accumulate ? grad[i] + g : g;
    }
}

// ---------------------------------------------------------------- batched GEMM

template <typename R, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    gemm_kernel(const GemmOp<R>* __restrict__ ops, const GemmTile* __restrict__ tiles) {
    constexpr int TX = BN / TN, TY = BM / TM, NT = TX * TY;
    __shared__ cpx<R> As[BK][BM + 1];
    __shared__ cpx<R> Bs[BK][BN + 1];
    const GemmTile tl = tiles[blockIdx.x];
    const GemmOp<R> op = ops[tl.op];
    const int row0 = tl.tm * BM, col0 = tl.tn * BN;
    int kbeg = 0, kend = op.K;
    if (op.triA == 1) kend = min(kend, row0 + BM);
    if (op.triA == 2) kbeg = max(kbeg, row0);
    if (op.triB == 1) kbeg = max(kbeg, col0);
    if (op.triB == 2) kend = min(kend, col0 + BN);
    kbeg = (kbeg / BK) * BK;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    cpx<R> acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = mk<R>(0, 0);
    const cpx<R> zero = mk<R>(0, 0);
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        for (int e = threadIdx.x; e < BM * BK; e += NT) {
            int r, kk;
            if (!op.transA) { r = e % BM; kk = e / BM; }
            else { kk = e % BK; r = e / BK; }
            const int gr = row0 + r, gk = k0 + kk;
            cpx<R> v = zero;
            if (gr < op.M && gk < kend) {
                v = op.transA ? op.A[gk + gr * op.lda] : op.A[gr + gk * op.lda];
                if (op.d) v = v * op.d[gk];
            }
            As[kk][r] = v;
        }
        for (int e = threadIdx.x; e < BK * BN; e += NT) {
            int c, kk;
            if (!op.transB) { kk = e % BK; c = e / BK; }
            else { c = e % BN; kk = e / BN; }
            const int gc = col0 + c, gk = k0 + kk;
            cpx<R> v = zero;
            if (gc < op.N && gk < kend) v = op.transB ? op.B[gc + gk * op.ldb] : op.B[gk + gc * op.ldb];
            Bs[kk][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            cpx<R> a[TM], bb[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[kk][ty + i * TY];
#pragma unroll
            for (int j = 0; j < TN; ++j) bb[j] = Bs[kk][tx + j * TX];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) cfma(acc[i][j], a[i], bb[j]);
        }
        __syncthreads();
    }
    const cpx<R> alpha = mk(op.alpha_re, op.alpha_im), beta = mk(op.beta_re, op.beta_im);
    const bool useBeta = (op.beta_re != R(0) || op.beta_im != R(0));
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int r = row0 + ty + i * TY;
        if (r >= op.M) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int c = col0 + tx + j * TX;
            if (c >= op.N || (op.lowerC && r < c)) continue;
            cpx<R>* cp = op.C + r + c * op.ldc;
            cpx<R> out = alpha * acc[i][j];
            if (useBeta) out += beta * (*cp);
            *cp = out;
        }
    }
}

// ---------------------------------------------------------------- front assembly

template <typename R>
__global__ void __launch_bounds__(kThreads) assemble_kernel(const FactorFront<R>* __restrict__ fronts,
                                                            const int* __restrict__ list, AssemblyParams ap) {
    const FactorFront<R> f = fronts[list[blockIdx.x]];
    const StencilParams& sp = ap.sp;
    const int nx = sp.nx, nxy = sp.nx * sp.ny;
    const int* ndToNat = ap.tabs.ndToNat[f.cls];
    const int* nbr = ap.tabs.nbrRows[f.cls];
    const int64_t ld = f.s + f.u;
    const z64 omega = mk(sp.omega, ap.damping);
    const z64* s3a = ap.s3a + f.s3aOff;
    const z64* is3a = ap.is3a + f.s3aOff;
    for (int j = threadIdx.x; j < f.s; j += blockDim.x) {
        const int col = f.ndOff + j;
        const int pn = ndToNat[col];
        const int xy = pn % nxy, vl = pn / nxy;
        const int x = xy % nx, y = xy / nx;
        const int z = sp.nz - 1 - (f.vOffset + vl);
        const double alpha = ap.vel[xy + (int64_t)z * nxy];
        const Terms t = StencilAt(sp, x, y, s3a[vl + 1], is3a[vl], is3a[vl + 1], is3a[vl + 2], omega, alpha);
        cpx<R>* colp = f.L + j * ld;
        colp[j] = ccast<R>(t.c);
        const z64 vals[6] = {t.xL, t.xR, t.yL, t.yR, t.vL, t.vR};
        const int* rows = nbr + (int64_t)col * 6;
#pragma unroll
        for (int n = 0; n < 6; ++n) {
            const int row = rows[n];
            if (row >= 0) colp[row] = ccast<R>(-vals[n]);
        }
    }
}

// ---------------------------------------------------------------- extend-add

template <typename R>
__global__ void __launch_bounds__(kThreads) extend_add_kernel(const FactorFront<R>* __restrict__ fronts,
                                                              const int2* __restrict__ tasks) {
    const int2 task = tasks[blockIdx.x];
    const FactorFront<R> ch = fronts[task.x];
    const FactorFront<R> p = fronts[ch.parent];
    const int b1 = min(task.y + 32, ch.u);
    const int64_t ldp = p.s + p.u;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, nw = blockDim.x / 32;
    for (int b = task.y + warp; b < b1; b += nw) {
        const int rb = ch.rel[b];
        const cpx<R>* ucol = ch.U + (int64_t)b * ch.u;
        if (rb < p.s) {
            cpx<R>* dst = p.L + rb * ldp;
            for (int a = b + lane; a < ch.u; a += 32) dst[ch.rel[a]] += ucol[a];
        } else {
            cpx<R>* dst = p.U + (int64_t)(rb - p.s) * p.u - p.s;
            for (int a = b + lane; a < ch.u; a += 32) dst[ch.rel[a]] += ucol[a];
        }
    }
}

// ---------------------------------------------------------------- LDL^T blocks

// Factor the b x b diagonal block at (J,J): unit L, pivots D, and inv(L_JJ)
// written into G's diagonal block.
template <typename R>
__global__ void __launch_bounds__(kThreads) ldl_diag_kernel(const FactorFront<R>* __restrict__ fronts,
                                                            const int* __restrict__ list, int J, int* status) {
    __shared__ cpx<R> A[kNB][kNB + 1];
    __shared__ cpx<R> X[kNB][kNB + 1];
    __shared__ cpx<R> w[kNB];
    const FactorFront<R> f = fronts[list[blockIdx.x]];
    const int b = min(kNB, f.s - J);
    const int64_t ld = f.s + f.u;
    cpx<R>* Lb = f.L + J + J * ld;
    const int tid = threadIdx.x;
    const cpx<R> zero = mk<R>(0, 0), one = mk<R>(1, 0);
    for (int e = tid; e < b * b; e += blockDim.x) {
        const int i = e % b, j = e / b;
        A[i][j] = (i >= j) ? Lb[i + j * ld] : zero;
    }
    __syncthreads();
    for (int j = 0; j < b; ++j) {
        const cpx<R> d = A[j][j];
        if (tid == 0 && ((d.re == R(0) && d.im == R(0)) || !(d.re == d.re) || !(d.im == d.im))) atomicOr(status, 1);
        const cpx<R> dinv = cinv(d);
        if (tid > j && tid < b) {
            w[tid] = A[tid][j];
            A[tid][j] = A[tid][j] * dinv;
        }
        __syncthreads();
        for (int e = tid; e < b * b; e += blockDim.x) {
            const int i = e % b, c = e / b;
            if (c > j && i >= c) A[i][c] -= A[i][j] * w[c];
        }
        __syncthreads();
    }
    for (int e = tid; e < b * b; e += blockDim.x) {
        const int i = e % b, j = e / b;
        Lb[i + j * ld] = (i > j) ? A[i][j] : (i == j ? one : zero);
    }
    if (tid < b) f.D[J + tid] = A[tid][tid];
    if (tid < b) {
        const int c = tid;
        for (int i = 0; i < b; ++i) X[i][c] = (i == c) ? one : zero;
        for (int i = c + 1; i < b; ++i) {
            cpx<R> acc = zero;
            for (int m = c; m < i; ++m) cfma(acc, A[i][m], X[m][c]);
            X[i][c] = -acc;
        }
    }
    __syncthreads();
    cpx<R>* Gb = f.G + J + J * (int64_t)f.ldg;
    for (int e = tid; e < b * b; e += blockDim.x) {
        const int i = e % b, j = e / b;
        Gb[i + j * (int64_t)f.ldg] = X[i][j];
    }
}

// L[r, J:J+b] := F[r, J:J+b] inv(L_JJ)^T inv(D_J) for a row tile below the block.
template <typename R>
__global__ void __launch_bounds__(kThreads) ldl_trsm_kernel(const FactorFront<R>* __restrict__ fronts,
                                                            const int2* __restrict__ tasks, int J) {
    constexpr int RT = kTrsmRows;
    __shared__ cpx<R> Li[kNB][kNB + 1];
    __shared__ cpx<R> Dinv[kNB];
    __shared__ cpx<R> Ar[RT][kNB + 1];
    const int2 task = tasks[blockIdx.x];
    const FactorFront<R> f = fronts[task.x];
    const int b = min(kNB, f.s - J);
    const int64_t ld = f.s + f.u;
    const int r0 = task.y;
    const int rows = min(RT, f.s + f.u - r0);
    const int tid = threadIdx.x;
    for (int e = tid; e < b * b; e += blockDim.x) {
        const int i = e % b, j = e / b;
        Li[i][j] = f.G[(J + i) + (J + j) * (int64_t)f.ldg];
    }
    if (tid < b) Dinv[tid] = cinv(f.D[J + tid]);
    for (int e = tid; e < rows * b; e += blockDim.x) {
        const int i = e % rows, m = e / rows;
        Ar[i][m] = f.L[(r0 + i) + (J + m) * ld];
    }
    __syncthreads();
    for (int e = tid; e < rows * b; e += blockDim.x) {
        const int i = e % rows, c = e / rows;
        cpx<R> acc = mk<R>(0, 0);
        for (int m = 0; m <= c; ++m) cfma(acc, Ar[i][m], Li[c][m]);
        f.L[(r0 + i) + (J + c) * ld] = acc * Dinv[c];
    }
}

// ---------------------------------------------------------------- GMRES vectors

constexpr int kReduceMaxBlocks = 1184;  // 8 per SM on 148 SMs

__global__ void norms_partial_kernel(const z64* __restrict__ w, int64_t npoints, int k, double* partial) {
    extern __shared__ double red[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    double acc = 0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.y + ty; p < npoints; p += (int64_t)gridDim.x * blockDim.y)
        acc += cabs2(w[p * k + tx]);
    red[ty * blockDim.x + tx] = acc;
    __syncthreads();
    for (int s = blockDim.y / 2; s > 0; s >>= 1) {
        if (ty < s) red[ty * blockDim.x + tx] += red[(ty + s) * blockDim.x + tx];
        __syncthreads();
    }
    if (ty == 0) partial[blockIdx.x * (int64_t)k + tx] = red[tx];
}

__global__ void sum_partial_real_kernel(const double* partial, int nblocks, int k, double* out, int sqrtOut) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= k) return;
    double acc = 0;
    for (int b = 0; b < nblocks; ++b) acc += partial[(int64_t)b * k + r];
    out[r] = sqrtOut ? sqrt(acc) : acc;
}

__global__ void mgs_step_kernel(z64* __restrict__ w, const z64* __restrict__ vprev, const z64* __restrict__ hprev,
                                const z64* __restrict__ vnext, int64_t npoints, int k, z64* partial) {
    extern __shared__ z64 redc[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const z64 h = vprev ? hprev[tx] : mk(0.0, 0.0);
    z64 acc = mk(0.0, 0.0);
    for (int64_t p = blockIdx.x * (int64_t)blockDim.y + ty; p < npoints; p += (int64_t)gridDim.x * blockDim.y) {
        const int64_t e = p * k + tx;
        z64 wv = w[e];
        if (vprev) {
            wv -= h * vprev[e];
            w[e] = wv;
        }
        if (vnext) {
            const z64 vv = vnext[e];
            acc += mk(vv.re * wv.re + vv.im * wv.im, vv.re * wv.im - vv.im * wv.re);  // conj(v) w
        }
    }
    if (!vnext) return;
    redc[ty * blockDim.x + tx] = acc;
    __syncthreads();
    for (int s = blockDim.y / 2; s > 0; s >>= 1) {
        if (ty < s) redc[ty * blockDim.x + tx] += redc[(ty + s) * blockDim.x + tx];
        __syncthreads();
    }
    if (ty == 0) partial[blockIdx.x * (int64_t)k + tx] = redc[tx];
}

__global__ void sum_partial_complex_kernel(const z64* partial, int nblocks, int k, z64* out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= k) return;
    z64 acc = mk(0.0, 0.0);
    for (int b = 0; b < nblocks; ++b) acc += partial[(int64_t)b * k + r];
    out[r] = acc;
}

__global__ void scale_columns_kernel(const z64* __restrict__ w, const double* __restrict__ s, z64* __restrict__ v,
                                     int64_t n, int k) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % k);
        const double inv = 1.0 / s[r];
        v[e] = inv * w[e];
    }
}

__global__ void combine_kernel(const z64* __restrict__ x0, const z64* __restrict__ V, int64_t vstride,
                               const z64* __restrict__ y, int j1, z64* __restrict__ x, int64_t n, int k) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % k);
        z64 acc = x0[e];
        for (int i = 0; i < j1; ++i) cfma(acc, y[i * k + r], V[i * vstride + e]);
        x[e] = acc;
    }
}

__global__ void axpy_columns_kernel(z64* __restrict__ w, const z64* __restrict__ v, const z64* __restrict__ h,
                                    int64_t n, int k) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % k);
        w[e] -= h[r] * v[e];
    }
}

inline dim3 ReduceBlockDim(int k) {
    int ty = 1;
    while (ty * 2 * k <= 256) ty *= 2;
    return dim3(k, ty);
}

unsigned ElementwiseGrid(int64_t n) { return (unsigned)std::min<int64_t>(CeilDiv(n, kThreads), 148 * 16); }

template <typename R, int BM, int BN, int BK, int TM, int TN>
void LaunchGemmCfg(const GemmOp<R>* ops, const GemmTile* tiles, int numTiles, cudaStream_t st) {
    constexpr int NT = (BM / TM) * (BN / TN);
    gemm_kernel<R, BM, BN, BK, TM, TN><<<numTiles, NT, 0, st>>>(ops, tiles);
    CUDA_LAUNCH_CHECK();
}

}  // namespace

// ---------------------------------------------------------------- host launchers

void LaunchHelmholtzApply(const z64* x, z64* y, const z64* b, const double* vel, const StencilParams& sp, int k,
                          cudaStream_t st) {
    dim3 grid(CeilDiv(sp.nx, kApplyTX), sp.ny, sp.nz);
    helmholtz_apply_kernel<<<grid, kThreads, 0, st>>>(x, y, b, vel, sp, k, 0, 0);
    CUDA_LAUNCH_CHECK();
}

void LaunchHelmholtzApplyPlanes(const z64* x, z64* y, const z64* b, const double* vel, const StencilParams& sp,
                                int k, int zFirst, int zCount, int zSlab, cudaStream_t st) {
    dim3 grid(CeilDiv(sp.nx, kApplyTX), sp.ny, zCount);
    helmholtz_apply_kernel<<<grid, kThreads, 0, st>>>(x, y, b, vel, sp, k, zFirst, zSlab);
    CUDA_LAUNCH_CHECK();
}

void LaunchVelocityGradient(const z64* U, const z64* Z, const double* vel, const StencilParams& sp, int k,
                            double* grad, int accumulate, cudaStream_t st) {
    const int64_t n = (int64_t)sp.nx * sp.ny * sp.nz;
    velocity_gradient_kernel<<<ElementwiseGrid(n), kThreads, 0, st>>>(U, Z, vel, sp, k, grad, accumulate);
    CUDA_LAUNCH_CHECK();
}

int GemmTileM(GemmShape) { return 64; }
int GemmTileN(GemmShape s) { return s == kGemmSquare ? 64 : 16; }

template <typename R>
void AppendGemmTiles(const GemmOp<R>& op, int opIndex, GemmShape shape, std::vector<GemmTile>& tiles) {
    const int BM = GemmTileM(shape), BN = GemmTileN(shape);
    if (op.M <= 0 || op.N <= 0) return;
    const int tmN = (int)CeilDiv(op.M, BM), tnN = (int)CeilDiv(op.N, BN);
    for (int tn = 0; tn < tnN; ++tn)
        for (int tm = 0; tm < tmN; ++tm) {
            if (op.lowerC && tm * BM + BM - 1 < tn * BN) continue;
            tiles.push_back(GemmTile{opIndex, tm, tn});
        }
}

template <typename R>
void LaunchGemm(const GemmOp<R>* ops, const GemmTile* tiles, int numTiles, GemmShape shape, cudaStream_t st) {
    if (numTiles <= 0) return;
    if (shape == kGemmSquare)
        LaunchGemmCfg<R, 64, 64, 8, 4, 4>(ops, tiles, numTiles, st);
    else
        LaunchGemmCfg<R, 64, 16, 16, 4, 1>(ops, tiles, numTiles, st);
}

template <typename R>
void LaunchAssemble(const FactorFront<R>* fronts, const int* list, int n, const AssemblyParams& ap,
                    cudaStream_t st) {
    if (n <= 0) return;
    assemble_kernel<R><<<n, kThreads, 0, st>>>(fronts, list, ap);
    CUDA_LAUNCH_CHECK();
}

template <typename R>
void LaunchExtendAdd(const FactorFront<R>* fronts, const int2* tasks, int n, cudaStream_t st) {
    if (n <= 0) return;
    extend_add_kernel<R><<<n, kThreads, 0, st>>>(fronts, tasks);
    CUDA_LAUNCH_CHECK();
}

template <typename R>
void LaunchLdlDiag(const FactorFront<R>* fronts, const int* list, int n, int J, int* status, cudaStream_t st) {
    if (n <= 0) return;
    ldl_diag_kernel<R><<<n, kThreads, 0, st>>>(fronts, list, J, status);
    CUDA_LAUNCH_CHECK();
}

template <typename R>
void LaunchLdlTrsm(const FactorFront<R>* fronts, const int2* tasks, int n, int J, cudaStream_t st) {
    if (n <= 0) return;
    ldl_trsm_kernel<R><<<n, kThreads, 0, st>>>(fronts, tasks, J);
    CUDA_LAUNCH_CHECK();
}

int ReduceBlocks(int64_t npoints, int k) {
    const dim3 bd = ReduceBlockDim(k);
    return (int)std::max<int64_t>(1, std::min<int64_t>(CeilDiv(npoints, bd.y), kReduceMaxBlocks));
}

void LaunchNormsPartial(const z64* w, int64_t npoints, int k, double* partial, cudaStream_t st) {
    const dim3 bd = ReduceBlockDim(k);
    norms_partial_kernel<<<ReduceBlocks(npoints, k), bd, sizeof(double) * bd.x * bd.y, st>>>(w, npoints, k, partial);
    CUDA_LAUNCH_CHECK();
}

void LaunchSumPartialReal(const double* partial, int nblocks, int k, double* out, int sqrtOut, cudaStream_t st) {
    sum_partial_real_kernel<<<CeilDiv(k, 64), 64, 0, st>>>(partial, nblocks, k, out, sqrtOut);
    CUDA_LAUNCH_CHECK();
}

void LaunchMgsStep(z64* w, const z64* v_prev, const z64* h_prev, const z64* v_next, int64_t npoints, int k,
                   z64* partial, cudaStream_t st) {
    const dim3 bd = ReduceBlockDim(k);
    mgs_step_kernel<<<ReduceBlocks(npoints, k), bd, sizeof(z64) * bd.x * bd.y, st>>>(w, v_prev, h_prev, v_next,
                                                                                     npoints, k, partial);
    CUDA_LAUNCH_CHECK();
}

void LaunchSumPartialComplex(const z64* partial, int nblocks, int k, z64* out, cudaStream_t st) {
    sum_partial_complex_kernel<<<CeilDiv(k, 64), 64, 0, st>>>(partial, nblocks, k, out);
    CUDA_LAUNCH_CHECK();
}

void LaunchScaleColumns(const z64* w, const double* s, z64* v, int64_t npoints, int k, cudaStream_t st) {
    const int64_t n = npoints * k;
    scale_columns_kernel<<<ElementwiseGrid(n), kThreads, 0, st>>>(w, s, v, n, k);
    CUDA_LAUNCH_CHECK();
}

void LaunchCombine(const z64* x0, const z64* V, int64_t vstride, const z64* y, int j1, z64* x, int64_t npoints,
                   int k, cudaStream_t st) {
    const int64_t n = npoints * k;
    combine_kernel<<<ElementwiseGrid(n), kThreads, 0, st>>>(x0, V, vstride, y, j1, x, n, k);
    CUDA_LAUNCH_CHECK();
}

void LaunchAxpyColumns(z64* w, const z64* v, const z64* h, int64_t npoints, int k, cudaStream_t st) {
    const int64_t n = npoints * k;
    axpy_columns_kernel<<<ElementwiseGrid(n), kThreads, 0, st>>>(w, v, h, n, k);
    CUDA_LAUNCH_CHECK();
}

#define PSP_INSTANTIATE(R)                                                                                      \
    template void AppendGemmTiles<R>(const GemmOp<R>&, int, GemmShape, std::vector<GemmTile>&);                \
    template void LaunchGemm<R>(const GemmOp<R>*, const GemmTile*, int, GemmShape, cudaStream_t);              \
    template void LaunchAssemble<R>(const FactorFront<R>*, const int*, int, const AssemblyParams&,             \
                                    cudaStream_t);                                                             \
    template void LaunchExtendAdd<R>(const FactorFront<R>*, const int2*, int, cudaStream_t);                   \
    template void LaunchLdlDiag<R>(const FactorFront<R>*, const int*, int, int, int*, cudaStream_t);           \
    template void LaunchLdlTrsm<R>(const FactorFront<R>*, const int2*, int, int, cudaStream_t);

PSP_INSTANTIATE(double)
PSP_INSTANTIATE(float)

}  // namespace psp_b200
