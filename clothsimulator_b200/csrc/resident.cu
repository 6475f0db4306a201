// Cluster-resident PCG: one thread-block cluster solves one sheet with the sheet's system
// held in the cluster's distributed shared memory for the whole solve.
//
// The batched loop of pcg.cu streams every sheet's matrix from HBM once per CG iteration
// (about 1.7 MB per 64x64 sheet, ~340 iterations per step).  A sheet of that size fits in
// the shared memory of an 8-CTA cluster (8 x 227 KB), so here each cluster
//   * takes the next sheet from a device work counter (persistent clusters; a sheet that
//     converges early frees its cluster at once, there is no batch-wide tail),
//   * copies its share of the sheet's SELL-32 panels into shared memory once,
//   * runs the same per-instance state machine as the batched loop (FP32 CG on the
//     correction system, FP64 dot products and norms, FP64 outer residual b - A dv64,
//     warm-start guard, inner and outer stopping tests) with the FP32 vectors in registers
//     (one thread per row) and the search direction p in shared memory, where the other
//     CTAs of the cluster read it through distributed shared memory (DSMEM),
//   * reduces dot products deterministically: warps by shuffle tree, warps of a CTA in
//     index order, CTAs of the cluster in rank order, every CTA summing the same partials
//     in the same order, so all CTAs take identical control decisions.
// Rows of a slice that does not fit the shared-memory panel budget are read from global
// memory (L2-resident at this working-set size) instead.
//
// Replaces the reference's per-cloth GPU solve (Cloth.cu:766-809) like pcg.cu does; the
// iteration is the same Jacobi-preconditioned CG (PhysicsHelper.cu:479-485 builds the
// scalar Jacobi preconditioner; here the 3x3 block inverse from the gather kernel).
#include <cooperative_groups.h>

#include "cs_internal.h"

namespace cg = cooperative_groups;

namespace {

constexpr int RES_NBUF = 3;  // rotating reduction buffers: a buffer is rewritten two syncs later

__device__ __forceinline__ double rwarp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float rwarp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ bool rfinite(double x) { return x == x && x < 1e300 && x > -1e300; }

// Cluster-wide sum of NV values.  fp32: partials and sums in float (the plain FP32 solver);
// otherwise double.  Ends with a cluster barrier; every thread of every CTA returns the
// same sums.  `red` holds RES_NBUF x CS_RES_MAX_CL x 2 doubles, `wsum` 32 x 2 doubles.
template <int NV>
__device__ __forceinline__ void cluster_sum(const cg::cluster_group& cl, int rank, int ncta, double* red, double* wsum,
                                            int& buf, double (&v)[NV], bool fp32) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; i++) v[i] = fp32 ? (double)rwarp_sum((float)v[i]) : rwarp_sum(v[i]);
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < NV; i++) wsum[2 * w + i] = v[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[NV];
#pragma unroll
        for (int i = 0; i < NV; i++) {
            if (fp32) {
                float a = 0.f;
                for (int j = 0; j < nw; j++) a += (float)wsum[2 * j + i];
                t[i] = (double)a;
            } else {
                double a = 0.0;
                for (int j = 0; j < nw; j++) a += wsum[2 * j + i];
                t[i] = a;
            }
        }
        double* slot = red + 2 * (buf * CS_RES_MAX_CL + rank);
        for (int c = 0; c < ncta; c++) {
            double* dst = cl.map_shared_rank(slot, c);
#pragma unroll
            for (int i = 0; i < NV; i++) dst[i] = t[i];
        }
    }
    cl.sync();
    const double* src = red + 2 * buf * CS_RES_MAX_CL;
#pragma unroll
    for (int i = 0; i < NV; i++) {
        if (fp32) {
            float a = 0.f;
            for (int c = 0; c < ncta; c++) a += (float)src[2 * c + i];
            v[i] = (double)a;
        } else {
            double a = 0.0;
            for (int c = 0; c < ncta; c++) a += src[2 * c + i];
            v[i] = a;
        }
    }
    buf = (buf + 1) % RES_NBUF;
}

}  // namespace

extern __shared__ __align__(16) unsigned char cs_res_smem[];

// Launch: cluster dimension (CL, 1, 1), blockDim = 32 x (slices per CTA, at most
// CS_RES_MAX_WARPS), dynamic shared memory = res_cap panels + one float4 per row slot.
// Grid: any number of whole clusters (persistent; each takes sheets until none is left).
__global__ void __launch_bounds__(CS_RES_MAX_WARPS * 32, 1) cs_resident_pcg_kernel(Batch B) {
    const DevParams P = *B.params;
    if (P.solver != CS_SOLVER_AUTO_DEV || B.n_resident == 0) return;  // uniform over the grid
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int ncta = (int)cl.num_blocks();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int cap = B.res_cap;
    const float* sm_panels = reinterpret_cast<const float*>(cs_res_smem);
    float4* sm_p = reinterpret_cast<float4*>(cs_res_smem + (size_t)cap * CS_PANEL_FLOATS * sizeof(float));
    __shared__ double red[RES_NBUF * CS_RES_MAX_CL * 2];
    __shared__ double wsum[64];
    __shared__ int sh_next;
    __shared__ const float4* prank[CS_RES_MAX_CL];
    if (threadIdx.x < ncta) prank[threadIdx.x] = cl.map_shared_rank(sm_p, (int)threadIdx.x);
    int buf = 0;
    const bool mixed = P.mixed != 0;
    const bool fp32 = !mixed;
    const int myslot = w * CS_SLICE + lane;
    __syncthreads();

    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            const int idx = atomicAdd(&B.loop[5], 1);
            for (int c = 0; c < ncta; c++) *cl.map_shared_rank(&sh_next, c) = idx;
        }
        cl.sync();
        const int idx = sh_next;
        if (idx >= B.n_resident) break;

        const int s = B.rlist[idx];
        const SheetDesc sh = B.sheets[s];
        const int* split = B.rsplit + sh.topo * (CS_RES_MAX_CL + 1);
        const int lo = split[rank], hi = split[rank + 1];
        int cta_p0 = 0, cta_p1 = 0;
        if (hi > lo) {
            cta_p0 = B.slices[sh.slice_off + lo].panel0;
            const SliceDesc& last = B.slices[sh.slice_off + hi - 1];
            cta_p1 = last.panel0 + last.width;
        }
        // this CTA's panels (contiguous) into shared memory, up to the budget
        {
            const int ncopy = min(cta_p1 - cta_p0, cap) * (CS_PANEL_FLOATS / 4);
            const float4* src = reinterpret_cast<const float4*>(B.A + (size_t)cta_p0 * CS_PANEL_FLOATS);
            float4* dst = reinterpret_cast<float4*>(cs_res_smem);
            for (int i = threadIdx.x; i < ncopy; i += blockDim.x) dst[i] = __ldg(src + i);
        }
        // this thread's row: slice lo + w, lane
        bool live = false;
        int width = 0, lp = 0, gp = 0, tp = 0, row = 0;
        if (lo + w < hi) {
            const SliceDesc d = B.slices[sh.slice_off + lo + w];
            live = lane < d.rows;
            width = d.width;
            gp = d.panel0;
            tp = d.tpanel0;
            lp = d.panel0 - cta_p0;
            if (live) row = B.rowmap[d.topo_slice * CS_SLICE + lane];
        }
        if (!live) width = 0;
        const bool in_smem = lp + width <= cap;
        const float* panels = in_smem ? sm_panels + (size_t)lp * CS_PANEL_FLOATS : B.A + (size_t)gp * CS_PANEL_FLOATS;
        const int g = sh.node_off + row;
        float Pi[9];
        float e[3] = {0.f, 0.f, 0.f}, r[3] = {0.f, 0.f, 0.f}, z[3] = {0.f, 0.f, 0.f};
        if (live) {
#pragma unroll
            for (int k = 0; k < 9; k++) Pi[k] = B.Pinv[9 * (size_t)g + k];
#pragma unroll
            for (int c = 0; c < 3; c++) r[c] = B.b[3 * g + c];
        } else {
#pragma unroll
            for (int k = 0; k < 9; k++) Pi[k] = 0.f;
        }
        const double bn = sqrt(B.inst[s].bnorm2);
        double rz = 0.0, rr = 0.0, pq = 0.0, res0 = bn, resnorm = -1.0, first_res = -1.0;
        float alpha = 0.f, beta = 0.f;
        int iters = 0, sweeps = 0, sweep_iters = 0, flags = 0, trips = 0;
        int phase = P.warm ? PH_RES : PH_INIT;

        while (phase != PH_FINISH) {
            if (++trips > P.loop_cap) {
                flags |= CS_IF_CAPPED;
                break;
            }
            if (phase == PH_RES) {
                // fold the FP32 correction into the FP64 solution, then r = b - A dv64 in FP64
                if (live) {
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        B.dv64[3 * g + c] += (double)e[c];
                        e[c] = 0.f;
                    }
                }
                cl.sync();
                double v[1] = {0.0};
                if (live) {
                    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
                    for (int k = 0; k < width; k++) {
                        const int col = __ldg(&B.tcol[(tp + k) * CS_SLICE + lane]) + sh.node_off;
                        const float* pn = panels + (size_t)k * CS_PANEL_FLOATS;
                        const float4 a0 = reinterpret_cast<const float4*>(pn)[lane];
                        const float4 a1 = reinterpret_cast<const float4*>(pn + 128)[lane];
                        const float a8 = pn[256 + lane];
                        const double d0 = B.dv64[3 * col], d1 = B.dv64[3 * col + 1], d2 = B.dv64[3 * col + 2];
                        y0 += (double)a0.x * d0 + (double)a0.y * d1 + (double)a0.z * d2;
                        y1 += (double)a0.w * d0 + (double)a1.x * d1 + (double)a1.y * d2;
                        y2 += (double)a1.z * d0 + (double)a1.w * d1 + (double)a8 * d2;
                    }
                    const double r0 = (double)B.b[3 * g] - y0, r1 = (double)B.b[3 * g + 1] - y1,
                                 r2 = (double)B.b[3 * g + 2] - y2;
                    r[0] = (float)r0;
                    r[1] = (float)r1;
                    r[2] = (float)r2;
                    v[0] = r0 * r0 + r1 * r1 + r2 * r2;
                }
                cluster_sum<1>(cl, rank, ncta, red, wsum, buf, v, false);
                const double res = sqrt(v[0]);
                resnorm = res;
                sweeps += 1;
                if (sweeps == 1) {
                    first_res = res;
                    if (P.warm && !(res <= bn)) {
                        // the warm start is worse than the zero guess: discard it
                        flags |= CS_IF_WARM_REJECTED;
                        res0 = bn;
                        phase = PH_INIT;
                        continue;
                    }
                }
                if (res <= P.tol * bn || bn == 0.0) {
                    flags |= CS_IF_CONVERGED;
                    phase = PH_FINISH;
                } else if (iters >= P.max_iters) {
                    flags |= CS_IF_CAPPED;
                    phase = PH_FINISH;
                } else if (mixed || rz == 0.0) {
                    res0 = res;
                    phase = PH_INIT;
                } else {
                    // plain FP32 CG stopped on its recursive residual and the FP64 check failed
                    flags |= CS_IF_CAPPED;
                    phase = PH_FINISH;
                }
            } else if (phase == PH_INIT) {
                if ((flags & CS_IF_WARM_REJECTED) && sweeps == 1 && live) {
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        B.dv64[3 * g + c] = 0.0;
                        r[c] = B.b[3 * g + c];
                    }
                }
                z[0] = Pi[0] * r[0] + Pi[1] * r[1] + Pi[2] * r[2];
                z[1] = Pi[3] * r[0] + Pi[4] * r[1] + Pi[5] * r[2];
                z[2] = Pi[6] * r[0] + Pi[7] * r[1] + Pi[8] * r[2];
                double v[2];
                if (mixed) {
                    v[0] = (double)r[0] * z[0] + (double)r[1] * z[1] + (double)r[2] * z[2];
                    v[1] = (double)r[0] * r[0] + (double)r[1] * r[1] + (double)r[2] * r[2];
                } else {
                    v[0] = (double)(r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
                    v[1] = (double)(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                }
                cluster_sum<2>(cl, rank, ncta, red, wsum, buf, v, fp32);
                rz = v[0];
                rr = v[1];
                beta = 0.f;
                sweep_iters = 0;
                phase = (rz > 0.0 && rfinite(rz)) ? PH_CG : PH_RES;
            } else {
                // PH_CG: p = z + beta p, q = A p, alpha, e += alpha p, r -= alpha q, z = P^-1 r, beta
                float p[3] = {z[0], z[1], z[2]};
                if (beta != 0.f) {
                    const float4 po = sm_p[myslot];
                    p[0] = __fmaf_rn(beta, po.x, p[0]);
                    p[1] = __fmaf_rn(beta, po.y, p[1]);
                    p[2] = __fmaf_rn(beta, po.z, p[2]);
                }
                if (live) sm_p[myslot] = make_float4(p[0], p[1], p[2], 0.f);
                cl.sync();
                float q0 = 0.f, q1 = 0.f, q2 = 0.f;
                for (int k = 0; k < width; k++) {
                    const uint32_t code = __ldg(reinterpret_cast<const uint32_t*>(B.rcode) + (tp + k) * CS_SLICE + lane);
                    const float* pn = panels + (size_t)k * CS_PANEL_FLOATS;
                    const float4 a0 = reinterpret_cast<const float4*>(pn)[lane];
                    const float4 a1 = reinterpret_cast<const float4*>(pn + 128)[lane];
                    const float a8 = pn[256 + lane];
                    const int ork = (int)(code >> 16), osl = (int)(code & 0xffffu);
                    const float4 pv = (ork == rank) ? sm_p[osl] : prank[ork][osl];
                    q0 += a0.x * pv.x + a0.y * pv.y + a0.z * pv.z;
                    q1 += a0.w * pv.x + a1.x * pv.y + a1.y * pv.z;
                    q2 += a1.z * pv.x + a1.w * pv.y + a8 * pv.z;
                }
                double v1[1];
                if (mixed)
                    v1[0] = (double)p[0] * q0 + (double)p[1] * q1 + (double)p[2] * q2;
                else
                    v1[0] = (double)(p[0] * q0 + p[1] * q1 + p[2] * q2);
                if (!live) v1[0] = 0.0;
                cluster_sum<1>(cl, rank, ncta, red, wsum, buf, v1, fp32);
                const double sum = v1[0];
                alpha = mixed ? (float)(rz / sum) : (float)rz / (float)sum;
                if (!(sum > 0.0) || !rfinite((double)alpha)) {
                    alpha = 0.f;
                    flags |= CS_IF_BREAKDOWN;
                }
                pq = sum;
                e[0] = __fmaf_rn(alpha, p[0], e[0]);
                e[1] = __fmaf_rn(alpha, p[1], e[1]);
                e[2] = __fmaf_rn(alpha, p[2], e[2]);
                r[0] = __fmaf_rn(-alpha, q0, r[0]);
                r[1] = __fmaf_rn(-alpha, q1, r[1]);
                r[2] = __fmaf_rn(-alpha, q2, r[2]);
                z[0] = Pi[0] * r[0] + Pi[1] * r[1] + Pi[2] * r[2];
                z[1] = Pi[3] * r[0] + Pi[4] * r[1] + Pi[5] * r[2];
                z[2] = Pi[6] * r[0] + Pi[7] * r[1] + Pi[8] * r[2];
                double v[2];
                if (mixed) {
                    v[0] = (double)r[0] * z[0] + (double)r[1] * z[1] + (double)r[2] * z[2];
                    v[1] = (double)r[0] * r[0] + (double)r[1] * r[1] + (double)r[2] * r[2];
                } else {
                    v[0] = (double)(r[0] * z[0] + r[1] * z[1] + r[2] * z[2]);
                    v[1] = (double)(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                }
                if (!live) v[0] = v[1] = 0.0;
                cluster_sum<2>(cl, rank, ncta, red, wsum, buf, v, fp32);
                float nb = mixed ? (float)(v[0] / rz) : (float)v[0] / (float)rz;
                rz = v[0];
                rr = v[1];
                iters += 1;
                sweep_iters += 1;
                const double rn = sqrt(rr);
                bool stop;
                if (mixed)
                    stop = rn <= P.inner_tol * res0 || rn <= 0.5 * P.tol * bn || sweep_iters >= P.sweep_cap;
                else
                    stop = rn <= P.tol * bn;
                if (!rfinite((double)nb) || !(rz > 0.0) || (flags & CS_IF_BREAKDOWN)) {
                    nb = 0.f;
                    stop = true;
                    flags |= CS_IF_BREAKDOWN;
                }
                beta = nb;
                if (stop || iters >= P.max_iters) phase = PH_RES;
            }
        }
        if (live && trips > P.loop_cap) {
#pragma unroll
            for (int c = 0; c < 3; c++) B.dv64[3 * g + c] += (double)e[c];
        }
        if (rank == 0 && threadIdx.x == 0) {
            InstState& I = B.inst[s];
            I.rz = rz;
            I.rr = rr;
            I.pq = pq;
            I.res0 = res0;
            I.resnorm = resnorm;
            I.first_res = first_res;
            I.alpha = alpha;
            I.beta = beta;
            I.iters = iters;
            I.sweeps = sweeps;
            I.sweep_iters = sweep_iters;
            I.flags = flags;
            I.phase = PH_DONE;
        }
        cl.sync();  // shared data of this sheet no longer read by any CTA
    }
}
