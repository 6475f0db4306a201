// Batched preconditioned conjugate gradients with per-instance convergence, FP32 vectors
// and SpMV, FP64 dot products and an FP64 outer residual (iterative refinement).
//
// Replaces the reference's GPU solve (Cloth.cu:766-809: cuSPARSE COO SpMV + cuBLAS, four
// host round trips per iteration, one cloth at a time) by one loop over all sheets.  Every
// instance (sheet) runs its own state machine (InstPhase); one trip of the loop runs four
// kernels over all slices, and each instance advances by one micro-step:
//
//   cs_spmv_kernel    PH_CG : p_new = z + beta p_old (fused), q = A p_new, partial p.q
//                     PH_RES: r = b - A (dv64 + e) in FP64, partial ||r||^2
//   cs_reduce1_kernel PH_CG : alpha = rz / pq
//                     PH_RES: accept (PH_FINISH) or go on with a new sweep (PH_INIT)
//   cs_vector_kernel  PH_CG : e += alpha p, r -= alpha q, z = P^-1 r, partials r.z, r.r
//                     PH_INIT / PH_FINISH: dv64 += e, e = 0 (and z, r.z for a new sweep)
//   cs_reduce2_kernel PH_CG : beta, inner stopping test; the last block counts unfinished
//                     instances and sets the CUDA-graph while-loop condition.
//
// Mixed precision uses reliable updates (Sleijpen and van der Vorst, 1996): a sweep ends when
// the recursive residual fell by inner_tol, the FP64 residual b - A dv64 replaces r, and CG
// goes on with the same search direction (beta = r.z / the previous iteration's r.z) instead
// of restarting from p = z, which would discard the Krylov space built so far.  It restarts
// when the replaced residual had drifted from the FP64 one by more than CS_RELIABLE_DRIFT of
// its norm: the kept direction would then no longer be conjugate to the new residual's.
//
// Reductions are deterministic: per-slice partials (one warp per slice), then one block per
// instance summing its slices in a fixed order.  p is double-buffered by loop-trip parity.
#include "cs_internal.h"

namespace {

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (blockDim.x == 128).
template <class T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
    v = warp_sum(v);
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) sh[w] = v;
    __syncthreads();
    T t = sh[0] + sh[1];
    t += sh[2] + sh[3];
    __syncthreads();
    return t;
}

// Deterministic block sums of two values (blockDim.x == CS_REDUCE_THREADS): warp butterflies,
// then the warps' partials in warp order.
template <class T>
__device__ __forceinline__ void block_sum2(T& a, T& b, T* sh) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh[2 * w] = a;
        sh[2 * w + 1] = b;
    }
    __syncthreads();
    a = sh[0];
    b = sh[1];
#pragma unroll
    for (int k = 1; k < CS_REDUCE_THREADS / 32; k++) {
        a += sh[2 * k];
        b += sh[2 * k + 1];
    }
    __syncthreads();
}

__device__ __forceinline__ bool finite_d(double x) { return x == x && x < 1e300 && x > -1e300; }

}  // namespace

// One slice of the batched SpMV (PH_CG: the CG product with the fused direction update; PH_RES:
// the FP64 residual).  UNROLL: slots whose loads are issued together; the sums still run in slot
// order, so every launch shape gives the same bits.
template <int UNROLL>
__device__ __forceinline__ void spmv_slice(const Batch& B, int slice, int lane) {
    const SliceDesc sd = B.slices[slice];
    const InstState& I = B.inst[sd.sheet];
    const int ph = I.phase;
    if (ph != PH_CG && ph != PH_RES) return;
    const bool mixed = B.params->mixed != 0;
    const int node_off = B.sheets[sd.sheet].node_off;
    const bool live = lane < sd.rows;
    const int row = sd.row0 + (live ? B.rowmap[sd.topo_slice * CS_SLICE + lane] : 0);
    if (ph == PH_CG) {
        const float beta = I.beta;
        const int par = B.loop[0] & 1;
        const float* __restrict__ pOld = par ? B.pB : B.pA;
        float* __restrict__ pNew = par ? B.pA : B.pB;
        const float* __restrict__ z = B.z;
        float y0 = 0.f, y1 = 0.f, y2 = 0.f;
        double dd = 0.0;
        float df = 0.f;
        if (live) {
#pragma unroll UNROLL
            for (int k = 0; k < sd.width; k++) {
                const int col = __ldg(&B.tcol[(sd.tpanel0 + k) * CS_SLICE + lane]) + node_off;
                const float* panel = B.A + (size_t)(sd.panel0 + k) * CS_PANEL_FLOATS;
                const float4 a0 = __ldg(reinterpret_cast<const float4*>(panel) + lane);
                const float4 a1 = __ldg(reinterpret_cast<const float4*>(panel + 128) + lane);
                const float a8 = __ldg(panel + 256 + lane);
                float p0 = z[3 * col], p1 = z[3 * col + 1], p2 = z[3 * col + 2];
                if (beta != 0.f) {
                    p0 = __fmaf_rn(beta, pOld[3 * col], p0);
                    p1 = __fmaf_rn(beta, pOld[3 * col + 1], p1);
                    p2 = __fmaf_rn(beta, pOld[3 * col + 2], p2);
                }
                y0 += a0.x * p0 + a0.y * p1 + a0.z * p2;
                y1 += a0.w * p0 + a1.x * p1 + a1.y * p2;
                y2 += a1.z * p0 + a1.w * p1 + a8 * p2;
            }
            if (B.xptr) {
                // proximity blocks outside the pattern (cs_set_proximities)
                for (int m = B.xptr[row]; m < B.xptr[row + 1]; m++) {
                    const int col = B.xcol[m];
                    const float* a = B.xval + 9 * (size_t)m;
                    float p0 = z[3 * col], p1 = z[3 * col + 1], p2 = z[3 * col + 2];
                    if (beta != 0.f) {
                        p0 = __fmaf_rn(beta, pOld[3 * col], p0);
                        p1 = __fmaf_rn(beta, pOld[3 * col + 1], p1);
                        p2 = __fmaf_rn(beta, pOld[3 * col + 2], p2);
                    }
                    y0 += a[0] * p0 + a[1] * p1 + a[2] * p2;
                    y1 += a[3] * p0 + a[4] * p1 + a[5] * p2;
                    y2 += a[6] * p0 + a[7] * p1 + a[8] * p2;
                }
            }
            float p0 = z[3 * row], p1 = z[3 * row + 1], p2 = z[3 * row + 2];
            if (beta != 0.f) {
                p0 = __fmaf_rn(beta, pOld[3 * row], p0);
                p1 = __fmaf_rn(beta, pOld[3 * row + 1], p1);
                p2 = __fmaf_rn(beta, pOld[3 * row + 2], p2);
            }
            pNew[3 * row] = p0;
            pNew[3 * row + 1] = p1;
            pNew[3 * row + 2] = p2;
            B.q[3 * row] = y0;
            B.q[3 * row + 1] = y1;
            B.q[3 * row + 2] = y2;
            if (mixed)
                dd = (double)p0 * y0 + (double)p1 * y1 + (double)p2 * y2;
            else
                df = p0 * y0 + p1 * y1 + p2 * y2;
        }
        if (mixed) {
            dd = warp_sum(dd);
            if (lane == 0) B.part[2 * slice] = dd;
        } else {
            df = warp_sum(df);
            if (lane == 0) B.part[2 * slice] = (double)df;
        }
    } else {
        double y0 = 0.0, y1 = 0.0, y2 = 0.0, sq = 0.0, dq = 0.0;
        if (live) {
#pragma unroll UNROLL
            for (int k = 0; k < sd.width; k++) {
                const int col = __ldg(&B.tcol[(sd.tpanel0 + k) * CS_SLICE + lane]) + node_off;
                const float* panel = B.A + (size_t)(sd.panel0 + k) * CS_PANEL_FLOATS;
                const float4 a0 = __ldg(reinterpret_cast<const float4*>(panel) + lane);
                const float4 a1 = __ldg(reinterpret_cast<const float4*>(panel + 128) + lane);
                const float a8 = __ldg(panel + 256 + lane);
                double d0 = B.dv64[3 * col] + (double)B.e[3 * col];
                double d1 = B.dv64[3 * col + 1] + (double)B.e[3 * col + 1];
                double d2 = B.dv64[3 * col + 2] + (double)B.e[3 * col + 2];
                y0 += (double)a0.x * d0 + (double)a0.y * d1 + (double)a0.z * d2;
                y1 += (double)a0.w * d0 + (double)a1.x * d1 + (double)a1.y * d2;
                y2 += (double)a1.z * d0 + (double)a1.w * d1 + (double)a8 * d2;
            }
            if (B.xptr) {
                for (int m = B.xptr[row]; m < B.xptr[row + 1]; m++) {
                    const int col = B.xcol[m];
                    const float* a = B.xval + 9 * (size_t)m;
                    const double d0 = B.dv64[3 * col] + (double)B.e[3 * col];
                    const double d1 = B.dv64[3 * col + 1] + (double)B.e[3 * col + 1];
                    const double d2 = B.dv64[3 * col + 2] + (double)B.e[3 * col + 2];
                    y0 += (double)a[0] * d0 + (double)a[1] * d1 + (double)a[2] * d2;
                    y1 += (double)a[3] * d0 + (double)a[4] * d1 + (double)a[5] * d2;
                    y2 += (double)a[6] * d0 + (double)a[7] * d1 + (double)a[8] * d2;
                }
            }
            double r0 = (double)B.b[3 * row] - y0, r1 = (double)B.b[3 * row + 1] - y1, r2 = (double)B.b[3 * row + 2] - y2;
            if (B.params->warm_scale && B.params->warm && !I.scaled) {
                // the warm start's scaling pass: d.b and d.r (d.A d = d.b - d.r) for its
                // Galerkin multiple
                const double d0 = B.dv64[3 * row] + (double)B.e[3 * row];
                const double d1 = B.dv64[3 * row + 1] + (double)B.e[3 * row + 1];
                const double d2 = B.dv64[3 * row + 2] + (double)B.e[3 * row + 2];
                sq = d0 * (double)B.b[3 * row] + d1 * (double)B.b[3 * row + 1] + d2 * (double)B.b[3 * row + 2];
                dq = d0 * r0 + d1 * r1 + d2 * r2;
            } else {
                // drift of the recursive residual it replaces
                const double q0 = r0 - (double)B.r[3 * row], q1 = r1 - (double)B.r[3 * row + 1],
                             q2 = r2 - (double)B.r[3 * row + 2];
                dq = q0 * q0 + q1 * q1 + q2 * q2;
                B.r[3 * row] = (float)r0;
                B.r[3 * row + 1] = (float)r1;
                B.r[3 * row + 2] = (float)r2;
                sq = r0 * r0 + r1 * r1 + r2 * r2;
            }
        }
        sq = warp_sum(sq);
        dq = warp_sum(dq);
        if (lane == 0) {
            B.part[2 * slice] = sq;
            B.part[2 * slice + 1] = dq;
        }
    }
}

// The batched SpMV kernel: each warp takes SPW consecutive slices.  Launch shapes (threads per
// block, SPW, UNROLL) are chosen per batch by cs_tune (ctx.cu); all give bitwise-identical output.
template <int SPW, int UNROLL>
__global__ void __launch_bounds__(512) cs_spmv_kernel_t(Batch B) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
#pragma unroll 1
    for (int i = 0; i < SPW; i++) {
        const int slice = warp * SPW + i;
        if (slice >= B.n_slices) return;
        spmv_slice<UNROLL>(B, slice, lane);
    }
}

// the candidates cs_tune times, in the order of CS_SPMV_CANDIDATES (cs_internal.h)
const SpmvShape kSpmvShapes[CS_SPMV_CANDIDATES] = {
    {64, 1, 1}, {128, 1, 1}, {256, 1, 1}, {512, 1, 1}, {64, 2, 1}, {128, 2, 1}, {256, 2, 1}, {512, 2, 1},
    {64, 4, 1}, {128, 4, 1}, {256, 4, 1}, {512, 4, 1}, {64, 1, 4}, {128, 1, 4}, {256, 1, 4}, {512, 1, 4},
    {64, 2, 4}, {128, 2, 4}, {256, 2, 4}, {512, 2, 4}, {64, 4, 4}, {128, 4, 4}, {256, 4, 4}, {512, 4, 4}};

void launchSpmvShape(const Batch& B, int shape, cudaStream_t st) {
    const SpmvShape& sh = kSpmvShapes[shape];
    const long long warps = (B.n_slices + sh.spw - 1) / sh.spw;
    const int grid = (int)((warps * 32 + sh.threads - 1) / sh.threads);
    if (grid <= 0) return;
#define CS_SPMV_LAUNCH(S, U) \
    if (sh.spw == S && sh.unroll == U) cs_spmv_kernel_t<S, U><<<grid, sh.threads, 0, st>>>(B);
    CS_SPMV_LAUNCH(1, 1) CS_SPMV_LAUNCH(2, 1) CS_SPMV_LAUNCH(4, 1) CS_SPMV_LAUNCH(1, 4) CS_SPMV_LAUNCH(2, 4)
    CS_SPMV_LAUNCH(4, 4)
#undef CS_SPMV_LAUNCH
}

// Sums of the two partials part[2 s], part[2 s + 1] over an instance's slices: double for the
// mixed solver, float for the plain FP32 solver.  Each thread takes every CS_REDUCE_THREADS-th
// slice, CS_REDUCE_UNROLL of them loaded together (16-byte loads of both partials) into as
// many running sums, added in a fixed order: the same bits on every run, and a sheet of
// 30,000 slices is summed in a few microseconds instead of one dependent load per slice.
#define CS_REDUCE_UNROLL 8
__device__ __forceinline__ void inst_sum2(const Batch& B, const SheetDesc& sh, bool mixed, double& s0, double& s1,
                                          double* shd, float* shf) {
    const double2* part = reinterpret_cast<const double2*>(B.part) + sh.slice_off;
    const int n = sh.n_slices, t = threadIdx.x;
    constexpr int T = CS_REDUCE_THREADS, U = CS_REDUCE_UNROLL;
    if (mixed) {
        double a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; u++) a[u] = b[u] = 0.0;
        int i = t;
        for (; i + (U - 1) * T < n; i += U * T) {
            double2 v[U];
#pragma unroll
            for (int u = 0; u < U; u++) v[u] = part[i + u * T];
#pragma unroll
            for (int u = 0; u < U; u++) {
                a[u] += v[u].x;
                b[u] += v[u].y;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (i + u * T < n) {
                const double2 v = part[i + u * T];
                a[u] += v.x;
                b[u] += v.y;
            }
        double x = a[0], y = b[0];
#pragma unroll
        for (int u = 1; u < U; u++) {
            x += a[u];
            y += b[u];
        }
        block_sum2(x, y, shd);
        s0 = x;
        s1 = y;
        return;
    }
    float a[U], b[U];
#pragma unroll
    for (int u = 0; u < U; u++) a[u] = b[u] = 0.f;
    int i = t;
    for (; i + (U - 1) * T < n; i += U * T) {
        double2 v[U];
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = part[i + u * T];
#pragma unroll
        for (int u = 0; u < U; u++) {
            a[u] += (float)v[u].x;
            b[u] += (float)v[u].y;
        }
    }
#pragma unroll
    for (int u = 0; u < U; u++)
        if (i + u * T < n) {
            const double2 v = part[i + u * T];
            a[u] += (float)v.x;
            b[u] += (float)v.y;
        }
    float x = a[0], y = b[0];
#pragma unroll
    for (int u = 1; u < U; u++) {
        x += a[u];
        y += b[u];
    }
    block_sum2(x, y, shf);
    s0 = (double)x;
    s1 = (double)y;
}

__global__ void __launch_bounds__(CS_REDUCE_THREADS) cs_reduce1_kernel(Batch B) {
    __shared__ double shd[2 * CS_REDUCE_THREADS / 32];
    __shared__ float shf[2 * CS_REDUCE_THREADS / 32];
    const int s = blockIdx.x;
    if (s == 0 && threadIdx.x == 0) {
        B.loop[1] = 0;
        B.loop[2] = 0;
    }
    InstState& I = B.inst[s];
    const int ph = I.phase;
    if (ph != PH_CG && ph != PH_RES) return;
    const DevParams& P = *B.params;
    const bool mixed = P.mixed != 0;
    const SheetDesc& sh = B.sheets[s];
    double sum, drift2;
    inst_sum2(B, sh, mixed || ph == PH_RES, sum, drift2, shd, shf);
    if (threadIdx.x != 0) return;
    if (ph == PH_RES && P.warm_scale && P.warm && !I.scaled) {
        // the warm start d becomes alpha d, alpha = d.b / d.A d (d.A d = d.b - d.r): the
        // multiple of d nearest to the solution in the energy norm; the guard then judges it
        const double db = sum, dad = sum - drift2, a = db / dad;
        I.scaled = 1;
        if (dad > 0.0 && finite_d(a)) {
            I.wscale = a;
            I.phase = PH_SCALE;
        } else {
            I.flags |= CS_IF_WARM_REJECTED;
            I.sweeps = 1;
            I.res0 = sqrt(I.bnorm2);
            I.phase = PH_INIT;
        }
        return;
    }
    if (!(ph == PH_RES && mixed)) drift2 = 0.0;
    if (ph == PH_CG) {
        float alpha;
        if (mixed)
            alpha = (float)(I.rz / sum);
        else
            alpha = (float)I.rz / (float)sum;
        if (!(sum > 0.0) || !finite_d((double)alpha)) {
            alpha = 0.f;
            I.flags |= CS_IF_BREAKDOWN;
        }
        I.pq = sum;
        I.alpha = alpha;
        return;
    }
    // PH_RES: FP64 residual norm of the current guess.
    const double res = sqrt(sum);
    const double bn = sqrt(I.bnorm2);
    I.resnorm = res;
    I.sweeps += 1;
    if (I.sweeps == 1) {
        I.first_res = res;
        if (P.warm && !(res <= bn)) {
            // The warm start is worse than the zero guess: discard it.
            I.flags |= CS_IF_WARM_REJECTED;
            I.res0 = bn;
            I.phase = PH_INIT;
            return;
        }
    }
    if (res <= P.tol * bn || bn == 0.0) {
        I.flags |= CS_IF_CONVERGED;
        I.phase = PH_FINISH;
    } else if (I.iters >= P.max_iters) {
        I.flags |= CS_IF_CAPPED;
        I.phase = PH_FINISH;
    } else if (mixed || I.rz == 0.0) {
        // mixed: a new CG sweep on the FP64 residual, continuing the search direction of the
        // last one if it ran; plain: the first sweep after a warm start
        I.res0 = res;
        I.cont = mixed && I.sweep_iters > 0 && !(I.flags & CS_IF_BREAKDOWN) && sqrt(drift2) <= CS_RELIABLE_DRIFT * res;
        I.phase = PH_INIT;
    } else {
        // Plain FP32 PCG stopped on its own recursive residual; the FP64 check above measured
        // its true residual, which FP32 rounding can keep above tol.  It ends here, unconverged.
        I.flags |= CS_IF_CAPPED;
        I.phase = PH_FINISH;
    }
}

// Warp w takes the rows of slice w's position in natural order: rows 32 k .. 32 k + 31 of the
// sheet for its k-th slice (a sheet has ceil(rows / 32) slices, the k-th holding as many rows
// as that range), so every vector access is contiguous; the partials per slice index sum to
// the same instance totals.
__global__ void __launch_bounds__(128) cs_vector_kernel(Batch B) {
    int slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (slice >= B.n_slices) return;
    const SliceDesc sd = B.slices[slice];
    const InstState& I = B.inst[sd.sheet];
    const int ph = I.phase;
    if (ph != PH_CG && ph != PH_INIT && ph != PH_FINISH && ph != PH_SCALE) return;
    const bool mixed = B.params->mixed != 0;
    const bool live = lane < sd.rows;
    const int row = sd.row0 + CS_SLICE * (slice - B.sheets[sd.sheet].slice_off) + (live ? lane : 0);
    if (ph == PH_SCALE) {
        if (live) {
            const double a = I.wscale;
#pragma unroll
            for (int c = 0; c < 3; c++) B.dv64[3 * row + c] *= a;
        }
        return;
    }
    double rz = 0.0, rr = 0.0;
    float rzf = 0.f, rrf = 0.f;
    if (live) {
        float r[3];
        if (ph == PH_CG) {
            const float alpha = I.alpha;
            const int par = B.loop[0] & 1;
            const float* __restrict__ pNew = par ? B.pA : B.pB;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                int i = 3 * row + c;
                B.e[i] = __fmaf_rn(alpha, pNew[i], B.e[i]);
                r[c] = __fmaf_rn(-alpha, B.q[i], B.r[i]);
                B.r[i] = r[c];
            }
        } else {
            const bool reset = (ph == PH_INIT) && (I.flags & CS_IF_WARM_REJECTED) && I.sweeps == 1;
            if (ph == PH_INIT && I.cont) {
                // the last direction is in this trip's old buffer (written two trips ago, the
                // FP64 residual trip between); the next trip reads its old p from the other one
                const int par = B.loop[0] & 1;
                const float* __restrict__ pLast = par ? B.pB : B.pA;
                float* __restrict__ pKeep = par ? B.pA : B.pB;
#pragma unroll
                for (int c = 0; c < 3; c++) pKeep[3 * row + c] = pLast[3 * row + c];
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                int i = 3 * row + c;
                if (reset) {
                    B.dv64[i] = 0.0;
                    r[c] = B.b[i];
                    B.r[i] = r[c];
                } else {
                    B.dv64[i] += (double)B.e[i];
                    r[c] = B.r[i];
                }
                B.e[i] = 0.f;
            }
            if (ph == PH_FINISH) r[0] = r[1] = r[2] = 0.f;
        }
        if (ph != PH_FINISH) {
            const float* Pi = B.Pinv + 9 * (size_t)row;
            float z0 = Pi[0] * r[0] + Pi[1] * r[1] + Pi[2] * r[2];
            float z1 = Pi[3] * r[0] + Pi[4] * r[1] + Pi[5] * r[2];
            float z2 = Pi[6] * r[0] + Pi[7] * r[1] + Pi[8] * r[2];
            B.z[3 * row] = z0;
            B.z[3 * row + 1] = z1;
            B.z[3 * row + 2] = z2;
            if (mixed) {
                rz = (double)r[0] * z0 + (double)r[1] * z1 + (double)r[2] * z2;
                rr = (double)r[0] * r[0] + (double)r[1] * r[1] + (double)r[2] * r[2];
            } else {
                rzf = r[0] * z0 + r[1] * z1 + r[2] * z2;
                rrf = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            }
        }
    }
    if (ph == PH_FINISH) return;
    if (mixed) {
        rz = warp_sum(rz);
        rr = warp_sum(rr);
    } else {
        rz = (double)warp_sum(rzf);
        rr = (double)warp_sum(rrf);
    }
    if (lane == 0) {
        B.part[2 * slice] = rz;
        B.part[2 * slice + 1] = rr;
    }
}

__global__ void __launch_bounds__(CS_REDUCE_THREADS) cs_reduce2_kernel(Batch B, cudaGraphConditionalHandle handle) {
    __shared__ double shd[2 * CS_REDUCE_THREADS / 32];
    __shared__ float shf[2 * CS_REDUCE_THREADS / 32];
    const int s = blockIdx.x;
    InstState& I = B.inst[s];
    const int ph = I.phase;
    const DevParams& P = *B.params;
    const bool mixed = P.mixed != 0;
    const SheetDesc& sh = B.sheets[s];
    if (ph == PH_CG || ph == PH_INIT) {
        double rz, rr;
        inst_sum2(B, sh, mixed, rz, rr, shd, shf);
        if (threadIdx.x == 0) {
            const double bn = sqrt(I.bnorm2);
            if (ph == PH_INIT) {
                float beta = 0.f;
                if (I.cont) {
                    // reliable update: r.z of the FP64 residual over the last iteration's r.z
                    const double bd = rz / I.rz_prev;
                    if (rz > 0.0 && finite_d(bd)) beta = (float)bd;
                    I.cont = 0;
                }
                I.rz = rz;
                I.rr = rr;
                I.beta = beta;
                I.sweep_iters = 0;
                I.phase = (rz > 0.0 && finite_d(rz)) ? PH_CG : PH_RES;
            } else {
                float beta = mixed ? (float)(rz / I.rz) : (float)rz / (float)I.rz;
                I.rz_prev = I.rz;
                I.rz = rz;
                I.rr = rr;
                I.iters += 1;
                I.sweep_iters += 1;
                const double rn = sqrt(rr);
                bool stop;
                if (mixed)
                    stop = rn <= P.inner_tol * I.res0 || rn <= 0.5 * P.tol * bn || I.sweep_iters >= P.sweep_cap;
                else
                    stop = rn <= P.tol * bn;
                if (!finite_d((double)beta) || !(rz > 0.0) || (I.flags & CS_IF_BREAKDOWN)) {
                    beta = 0.f;
                    stop = true;
                    I.flags |= CS_IF_BREAKDOWN;
                }
                I.beta = beta;
                if (stop || I.iters >= P.max_iters) I.phase = PH_RES;
            }
        }
    } else if (threadIdx.x == 0) {
        if (ph == PH_FINISH) I.phase = PH_DONE;
        else if (ph == PH_SCALE) I.phase = PH_RES;  // the residual of the scaled warm start
    }
    if (threadIdx.x == 0) {
        if (I.phase != PH_DONE && I.phase != PH_RESIDENT) atomicAdd(&B.loop[1], 1);
        __threadfence();
        int ticket = atomicAdd(&B.loop[2], 1);
        if (ticket == (int)gridDim.x - 1) {
            __threadfence();
            int remaining = atomicAdd(&B.loop[1], 0);
            int trips = B.loop[0] + 1;
            B.loop[0] = trips;
            B.loop[4] += 1;  // cumulative trips since load
            int go = (remaining > 0 && trips < P.loop_cap) ? 1 : 0;
            B.loop[3] = go;
            if (handle) cudaGraphSetConditional(handle, go);
        }
    }
}

// Start of a solve: per node, dv64 = warm start (or 0), e = 0, r = b, p buffers = 0.
__global__ void cs_solve_prologue_kernel(Batch B) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * B.N) return;
    const bool warm = B.params->warm != 0;
    B.dv64[i] = warm ? (double)B.warm[i] : 0.0;
    B.e[i] = 0.f;
    B.r[i] = B.b[i];
    B.pA[i] = 0.f;
    B.pB[i] = 0.f;
}

// Per instance: ||b||^2 from the assembly's slice partials, and the initial phase.
__global__ void __launch_bounds__(128) cs_solve_setup_kernel(Batch B) {
    __shared__ double shd[4];
    const int s = blockIdx.x;
    const SheetDesc& sh = B.sheets[s];
    double acc = 0.0;
    for (int i = threadIdx.x; i < sh.n_slices; i += blockDim.x) acc += B.part[2 * (sh.slice_off + i)];
    acc = block_sum(acc, shd);
    if (threadIdx.x == 0) {
        InstState& I = B.inst[s];
        I.bnorm2 = acc;
        I.rz = I.rz_prev = I.pq = I.rr = 0.0;
        I.cont = 0;
        I.res0 = sqrt(acc);
        I.resnorm = I.first_res = -1.0;
        I.alpha = I.beta = 0.f;
        I.sweep_iters = I.iters = I.sweeps = I.flags = 0;
        I.scaled = 0;
        I.wscale = 1.0;
        if (sh.resident && B.params->solver == CS_SOLVER_AUTO_DEV && !(B.sheet_prox && B.sheet_prox[s]))
            I.phase = PH_RESIDENT;  // solved by cs_resident_pcg_kernel before the loop runs
        else
            I.phase = B.params->warm ? PH_RES : PH_INIT;
        if (s == 0) {
            B.loop[0] = 0;
            B.loop[1] = 0;
            B.loop[2] = 0;
            B.loop[3] = 1;
            B.loop[5] = 0;
            B.loop[6] = 0;
        }
    }
}

// End of a step: dv = dv64, v += dv (Cloth.cu:690-692), x += dt v (Mesh.cu:226-231); the
// solution is kept as the next step's warm start.
__global__ void cs_advance_kernel(Batch B) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * B.N) return;
    float d = (float)B.dv64[i];
    B.dv[i] = d;
    B.warm[i] = d;
    if (B.params->advance) {
        float v = __fadd_rn(B.v[i], d);
        B.v[i] = v;
        const float x = B.x[i];
        B.x0[i] = x;  // Mesh::updatePositions (Mesh.cu:226-231)
        B.x[i] = __fadd_rn(x, __fmul_rn(B.params->dt, v));
    }
}

// y = A x for the inspection entry point cs_spmv (one warp per slice, FP32).
__global__ void __launch_bounds__(128) cs_spmv_plain_kernel(Batch B, const float* __restrict__ x, float* __restrict__ y) {
    int slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (slice >= B.n_slices) return;
    const SliceDesc sd = B.slices[slice];
    if (lane >= sd.rows) return;
    const int node_off = B.sheets[sd.sheet].node_off;
    const int row = sd.row0 + B.rowmap[sd.topo_slice * CS_SLICE + lane];
    float y0 = 0.f, y1 = 0.f, y2 = 0.f;
    for (int k = 0; k < sd.width; k++) {
        const int col = B.tcol[(sd.tpanel0 + k) * CS_SLICE + lane] + node_off;
        const float* panel = B.A + (size_t)(sd.panel0 + k) * CS_PANEL_FLOATS;
        const float4 a0 = reinterpret_cast<const float4*>(panel)[lane];
        const float4 a1 = reinterpret_cast<const float4*>(panel + 128)[lane];
        const float a8 = panel[256 + lane];
        const float p0 = x[3 * col], p1 = x[3 * col + 1], p2 = x[3 * col + 2];
        y0 += a0.x * p0 + a0.y * p1 + a0.z * p2;
        y1 += a0.w * p0 + a1.x * p1 + a1.y * p2;
        y2 += a1.z * p0 + a1.w * p1 + a8 * p2;
    }
    if (B.xptr) {
        for (int m = B.xptr[row]; m < B.xptr[row + 1]; m++) {
            const int col = B.xcol[m];
            const float* a = B.xval + 9 * (size_t)m;
            const float p0 = x[3 * col], p1 = x[3 * col + 1], p2 = x[3 * col + 2];
            y0 += a[0] * p0 + a[1] * p1 + a[2] * p2;
            y1 += a[3] * p0 + a[4] * p1 + a[5] * p2;
            y2 += a[6] * p0 + a[7] * p1 + a[8] * p2;
        }
    }
    y[3 * row] = y0;
    y[3 * row + 1] = y1;
    y[3 * row + 2] = y2;
}

// Measurement only: holds every instance in one phase with finite solver scalars so that a
// single solver kernel can be timed in isolation (cs_profile_kernels).
__global__ void cs_profile_setup_kernel(Batch B, int phase) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B.S) return;
    InstState& I = B.inst[s];
    I.phase = phase;
    I.alpha = 0.25f;
    I.beta = 0.5f;
    I.rz = 1.0;
}
