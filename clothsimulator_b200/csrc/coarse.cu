// Coarse-space correction of the batched PCG loop (pcg.cu).  No reference counterpart: the
// reference's GPU solve is Jacobi-PCG (Cloth.cu:766-809).
//
// Block-Jacobi PCG needs many iterations on a large sheet (1,700 on a 1,000 x 1,000 grid): the
// smooth error spans the sheet and the diagonal blocks cannot move it.  Each sheet's nodes are
// grouped into aggregates (its rest (u, v) coordinates binned into g x g cells, the non-empty
// cells), and the preconditioner becomes additive two-level,
//     z = D^-1 r + R^T A_c^-1 R r,
// R summing a vector over each aggregate (one value per aggregate and component) and
// A_c = R A R^T.  Per step: A_c is summed from per-pair contributor lists (a fixed order, so
// the result is deterministic) and inverted by Gauss-Jordan in FP32 -- one CTA with the matrix
// in shared memory up to CS_BC_SMALL_NC unknowns, else a cluster of CS_BC_CLUSTER CTAs with its
// rows spread over their shared memory and each pivot row read through distributed shared
// memory -- then symmetrised.  A_c is SPD (A is), so no pivoting is needed; the pivots are
// diagonal blocks of CS_BC_PB aggregates (CS_BC_KB rows, a twelfth of the barriers of scalar
// pivots), and a non-positive pivot inside one disables the sheet's correction for the step.  Per CG trip, after the vector
// update: R r (a block per aggregate), e_c = A_c^-1 R r (a warp per coarse row), then
// z += R^T e_c with the r.z and r.r partials recomputed (a warp per 32 rows in natural order,
// as cs_vector_kernel lays them out).  Sheets solved cluster-resident (their own coarse
// correction, resident.cu) and sheets with proximities (blocks outside the pattern) skip it.
#include <cooperative_groups.h>

#include "cs_internal.h"

namespace cg = cooperative_groups;

static_assert(CS_BC_MAX_NC <= 2 * CS_BC_THREADS, "a thread of the cluster inversion updates at most two columns");

namespace {

template <class T>
__device__ __forceinline__ T bc_warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The sheet takes the correction this step (independent of its phase).
__device__ __forceinline__ bool bc_sheet_on(const Batch& B, int s) {
    if (!B.params->coarse || !B.bc_agg) return false;
    if (B.sheets[s].bc_na <= 0) return false;
    if (B.sheet_prox && B.sheet_prox[s]) return false;
    return true;
}

// The sheet applies the correction in this trip: a CG iteration or a sweep start of the loop.
__device__ __forceinline__ bool bc_trip_on(const Batch& B, int s) {
    const int ph = B.inst[s].phase;
    return (ph == PH_CG || ph == PH_INIT) && bc_sheet_on(B, s) && B.bc_ok[s];
}

}  // namespace

// A_c of every sheet the loop solves: a warp per coarse pair (a, b) sums the 3x3 blocks of its
// contributor slots (lane-strided, then a butterfly: a fixed order) into rows 3a..3a+2,
// columns 3b..3b+2 of the sheet's dense coarse matrix (zeroed before).  Grid: x over pairs,
// y over sheets.
__global__ void __launch_bounds__(256) cs_bc_assemble_kernel(Batch B) {
    const int s = blockIdx.y;
    if (!bc_sheet_on(B, s) || B.inst[s].phase == PH_RESIDENT) return;
    const SheetDesc& sh = B.sheets[s];
    const int nc = 3 * sh.bc_na;
    float* M = B.bc_mat + sh.bc_mat_off;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int q = blockIdx.x * wpb + (threadIdx.x >> 5); q < sh.bc_npair; q += gridDim.x * wpb) {
        const int4 pr = B.bc_pair[sh.bc_pair_off + q];
        float a[9];
#pragma unroll
        for (int k = 0; k < 9; k++) a[k] = 0.f;
        for (int k = pr.z + lane; k < pr.w; k += 32) {
            const int slot = B.bc_contrib[k];
            const float* panel = B.A + (size_t)(sh.panel_off + (slot >> 5)) * CS_PANEL_FLOATS;
            const int l = slot & 31;
            const float4 a0 = reinterpret_cast<const float4*>(panel)[l];
            const float4 a1 = reinterpret_cast<const float4*>(panel + 128)[l];
            const float a8 = panel[256 + l];
            a[0] += a0.x;
            a[1] += a0.y;
            a[2] += a0.z;
            a[3] += a0.w;
            a[4] += a1.x;
            a[5] += a1.y;
            a[6] += a1.z;
            a[7] += a1.w;
            a[8] += a8;
        }
#pragma unroll
        for (int k = 0; k < 9; k++) a[k] = bc_warp_sum(a[k]);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 9; k++) M[(size_t)(3 * pr.x + k / 3) * nc + 3 * pr.y + k % 3] = a[k];
        }
    }
}

// In-place Gauss-Jordan inverse of a kn x kn SPD block (kn <= CS_BC_KB, row stride
// CS_BC_KB) in shared memory by one warp; false (the same in every lane) if a pivot is not
// positive.  Each lane reads its elements' old values before the warp writes the new ones.
__device__ bool bc_warp_inverse(float* D, int kn) {
    const int lane = threadIdx.x & 31;
    constexpr int PER = (CS_BC_KB * CS_BC_KB + 31) / 32;
    int ii[PER], jj[PER];
#pragma unroll
    for (int m = 0; m < PER; m++) {
        const int e = lane + 32 * m;
        ii[m] = e < kn * kn ? e / kn : -1;
        jj[m] = e < kn * kn ? e - ii[m] * kn : 0;
    }
    for (int p = 0; p < kn; p++) {
        const float piv = D[p * CS_BC_KB + p];
        if (!(piv > 0.f) || !isfinite(piv)) return false;
        const float ip = 1.0f / piv;
        float nv[PER];
#pragma unroll
        for (int m = 0; m < PER; m++) {
            const int i = ii[m], j = jj[m];
            nv[m] = 0.f;
            if (i >= 0) {
                const float a = D[i * CS_BC_KB + j], ci = D[i * CS_BC_KB + p], pj = D[p * CS_BC_KB + j];
                nv[m] = i == p ? (j == p ? ip : pj * ip) : (j == p ? -ci * ip : a - ci * (pj * ip));
            }
        }
        __syncwarp();
#pragma unroll
        for (int m = 0; m < PER; m++)
            if (ii[m] >= 0) D[ii[m] * CS_BC_KB + jj[m]] = nv[m];
        __syncwarp();
    }
    return true;
}

// t[r] = sum_q C[r][q] u[q] for four rows of 12 coefficients each (16-byte loads, the rows'
// chains independent); C rows 48 bytes apart.
__device__ __forceinline__ void bc_dot12x4(const float* C, const float (&u)[CS_BC_KB], float (&t)[4]) {
    static_assert(CS_BC_KB == 12, "four-aggregate pivot blocks");
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const float4* c4 = reinterpret_cast<const float4*>(C + r * CS_BC_KB);
        const float4 a = c4[0], b = c4[1], c = c4[2];
        float x = a.x * u[0];
        float y = a.y * u[1];
        x = __fmaf_rn(a.z, u[2], x);
        y = __fmaf_rn(a.w, u[3], y);
        x = __fmaf_rn(b.x, u[4], x);
        y = __fmaf_rn(b.y, u[5], y);
        x = __fmaf_rn(b.z, u[6], x);
        y = __fmaf_rn(b.w, u[7], y);
        x = __fmaf_rn(c.x, u[8], x);
        y = __fmaf_rn(c.y, u[9], y);
        x = __fmaf_rn(c.z, u[10], x);
        y = __fmaf_rn(c.w, u[11], y);
        t[r] = x + y;
    }
}

// out[t * ldo] = sum_v D[t][v] a[v * lda] for t < kn (one column of D^-1 A[K, :]); a full
// block's sums unrolled with their loads issued together.
__device__ __forceinline__ void bc_block_rows_times(const float* D, const float* a, int lda, int kn, float* out,
                                                    int ldo) {
    if (kn == CS_BC_KB) {
        float av[CS_BC_KB];
#pragma unroll
        for (int v = 0; v < CS_BC_KB; v++) av[v] = a[(size_t)v * lda];
#pragma unroll
        for (int t = 0; t < CS_BC_KB; t++) {
            const float* d = D + t * CS_BC_KB;
            float x = d[0] * av[0], y = d[1] * av[1];
#pragma unroll
            for (int v = 2; v < CS_BC_KB; v += 2) {
                x = __fmaf_rn(d[v], av[v], x);
                y = __fmaf_rn(d[v + 1], av[v + 1], y);
            }
            out[(size_t)t * ldo] = x + y;
        }
        return;
    }
    for (int t = 0; t < kn; t++) {
        float u = 0.f;
        for (int v = 0; v < kn; v++) u = __fmaf_rn(D[t * CS_BC_KB + v], a[(size_t)v * lda], u);
        out[(size_t)t * ldo] = u;
    }
}

// Gauss-Jordan inversion in place with pivot blocks of CS_BC_PB aggregates (CS_BC_KB rows: a
// twelfth of the barriers of scalar pivots) of an SPD matrix held by one CTA in shared memory
// (nc <= CS_BC_SMALL_NC), a block per sheet; the inverse is written symmetrised.  Per pivot
// block K (kn rows from k0): D = A[K, K] inverted by one warp, U = D^-1 A[K, :] with U[:, K] =
// D^-1, then every row i outside K gets A[i, :] -= A[i, K] U (the K columns: -A[i, K] D^-1) and
// rows K become U.  Thread t updates column t % nc of rows t / nc, t / nc + blockDim / nc, ...
__global__ void __launch_bounds__(CS_BC_THREADS) cs_bc_invert_small_kernel(Batch B) {
    extern __shared__ float bc_sm[];
    __shared__ int bad;
    const int s = blockIdx.x;
    if (!bc_sheet_on(B, s) || B.inst[s].phase == PH_RESIDENT) return;
    const SheetDesc& sh = B.sheets[s];
    const int nc = 3 * sh.bc_na;
    if (nc > CS_BC_SMALL_NC) return;
    float* M = bc_sm;
    float* colb = bc_sm + ((nc * nc + 3) & ~3);  // nc x CS_BC_KB: A[i, K], 16-byte aligned rows
    float* U = colb + CS_BC_KB * nc;             // CS_BC_KB x nc
    float* D = U + CS_BC_KB * nc;                // CS_BC_KB x CS_BC_KB
    const float* G = B.bc_mat + sh.bc_mat_off;
    const int n2 = nc * nc;
    for (int e = threadIdx.x; e < n2; e += blockDim.x) M[e] = G[e];
    if (threadIdx.x == 0) bad = 0;
    const int rs = blockDim.x / nc, j = threadIdx.x % nc, i0 = threadIdx.x / nc;
    const bool active = i0 < rs;  // threads beyond rs * nc idle in the update
    __syncthreads();
    for (int k0 = 0; k0 < nc; k0 += CS_BC_KB) {
        const int kn = min(CS_BC_KB, nc - k0);
        for (int e = threadIdx.x; e < kn * kn; e += blockDim.x) {
            const int a = e / kn, b = e - a * kn;
            D[a * CS_BC_KB + b] = M[(k0 + a) * nc + k0 + b];
        }
        for (int e = threadIdx.x; e < nc * CS_BC_KB; e += blockDim.x) {
            const int i = e / CS_BC_KB, t = e - i * CS_BC_KB;
            colb[e] = t < kn ? M[i * nc + k0 + t] : 0.f;
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            const bool ok = bc_warp_inverse(D, kn);
            if (threadIdx.x == 0 && !ok) bad = 1;
        }
        __syncthreads();
        if (bad) break;  // uniform: read after the barrier
        for (int q = threadIdx.x; q < nc; q += blockDim.x) {
            const int c = q - k0;
            if (c >= 0 && c < kn) {
                for (int t = 0; t < kn; t++) U[t * nc + q] = D[t * CS_BC_KB + c];
                continue;
            }
            bc_block_rows_times(D, M + (size_t)k0 * nc + q, nc, kn, U + q, nc);
        }
        __syncthreads();
        if (active) {
            float uj[CS_BC_KB];
#pragma unroll
            for (int t = 0; t < CS_BC_KB; t++) uj[t] = t < kn ? U[t * nc + j] : 0.f;
            const bool jk = j >= k0 && j < k0 + kn;
            for (int i = i0; i < nc; i += rs) {
                float v;
                if (i >= k0 && i < k0 + kn) v = U[(i - k0) * nc + j];
                else {
                    const float4* c4 = reinterpret_cast<const float4*>(colb + i * CS_BC_KB);
                    const float4 a = c4[0], b = c4[1], c = c4[2];
                    float x = a.x * uj[0], y = a.y * uj[1];
                    x = __fmaf_rn(a.z, uj[2], x);
                    y = __fmaf_rn(a.w, uj[3], y);
                    x = __fmaf_rn(b.x, uj[4], x);
                    y = __fmaf_rn(b.y, uj[5], y);
                    x = __fmaf_rn(b.z, uj[6], x);
                    y = __fmaf_rn(b.w, uj[7], y);
                    x = __fmaf_rn(c.x, uj[8], x);
                    y = __fmaf_rn(c.y, uj[9], y);
                    x = __fmaf_rn(c.z, uj[10], x);
                    y = __fmaf_rn(c.w, uj[11], y);
                    const float t = x + y;
                    v = jk ? -t : M[i * nc + j] - t;
                }
                M[i * nc + j] = v;
            }
        }
        __syncthreads();
    }
    __syncthreads();
    float* Inv = B.bc_inv + sh.bc_mat_off;
    if (!bad)
        for (int e = threadIdx.x; e < n2; e += blockDim.x) {
            const int i = e / nc, jj = e - i * nc;
            Inv[e] = 0.5f * (M[e] + M[jj * nc + i]);
        }
    if (threadIdx.x == 0) B.bc_ok[s] = bad ? 0 : 1;
}

// The same inversion of a larger coarse matrix (CS_BC_SMALL_NC < nc <= CS_BC_MAX_NC) by a
// cluster of CS_BC_CLUSTER CTAs, one cluster per sheet of B.bc_big: rank c holds the rows of
// pivot blocks c, c + CS_BC_CLUSTER, ... in shared memory.  Per pivot block its owner inverts
// D (one warp) and writes U and a validity flag into its buffer, one cluster barrier, then every
// other CTA copies the buffer from the owner's shared memory into its own (16-byte distributed
// shared memory loads) and all update their rows, thread t columns t and t + blockDim.  A CTA's
// buffer is overwritten (by its own copy or its own U) only after the barrier that follows
// every other CTA's copy from it, so one cluster barrier per pivot block suffices.  The raw
// inverse goes back to bc_mat, then (after a barrier) each CTA writes its rows of the
// symmetrised inverse.
__global__ void __launch_bounds__(CS_BC_THREADS) cs_bc_invert_cluster_kernel(Batch B) {
    extern __shared__ float bc_sm[];
    __shared__ int bad;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int s = B.bc_big[blockIdx.x / CS_BC_CLUSTER];
    // the same decision in every CTA of the cluster: all return, or none
    if (!bc_sheet_on(B, s) || B.inst[s].phase == PH_RESIDENT) return;
    const SheetDesc& sh = B.sheets[s];
    const int nc = 3 * sh.bc_na;
    if (nc <= CS_BC_SMALL_NC || nc > CS_BC_MAX_NC) return;
    const int nblk = (nc + CS_BC_KB - 1) / CS_BC_KB;              // only the last may be partial
    const int RM = CS_BC_KB * ((nblk + CS_BC_CLUSTER - 1) / CS_BC_CLUSTER);
    int R = 0;                                                     // this CTA's rows
    for (int kb = rank; kb < nblk; kb += CS_BC_CLUSTER) R += min(CS_BC_KB, nc - CS_BC_KB * kb);
    const int UB = (CS_BC_KB * nc + 1 + 3) & ~3;                   // U, the flag, padded to 16 bytes
    float* M = bc_sm;                                              // RM x nc
    float* lbuf = bc_sm + ((RM * nc + 3) & ~3);                    // UB
    float* colb = lbuf + UB;                                       // RM x CS_BC_KB: A[i, K]
    float* D = colb + RM * CS_BC_KB;                               // CS_BC_KB x CS_BC_KB
    float* G = B.bc_mat + sh.bc_mat_off;
    auto grow = [&](int li) { return CS_BC_KB * (rank + CS_BC_CLUSTER * (li / CS_BC_KB)) + li % CS_BC_KB; };
    for (int e = threadIdx.x; e < R * nc; e += blockDim.x) {
        const int li = e / nc, j = e - li * nc;
        M[e] = G[(size_t)grow(li) * nc + j];
    }
    if (threadIdx.x == 0) bad = 0;
    cluster.sync();  // every CTA has started and loaded its rows before remote reads
    const int j0 = threadIdx.x, j1 = threadIdx.x + blockDim.x;
    for (int kb = 0; kb < nblk; kb++) {
        const int owner = kb % CS_BC_CLUSTER, k0 = CS_BC_KB * kb, kn = min(CS_BC_KB, nc - k0);
        for (int e = threadIdx.x; e < RM * CS_BC_KB; e += blockDim.x) {
            const int li = e / CS_BC_KB, t = e - li * CS_BC_KB;
            colb[e] = (li < R && t < kn) ? M[li * nc + k0 + t] : 0.f;  // rows and columns past the data: 0
        }
        if (rank == owner) {
            const int l0 = CS_BC_KB * (kb / CS_BC_CLUSTER);
            for (int e = threadIdx.x; e < kn * kn; e += blockDim.x) {
                const int a = e / kn, b = e - a * kn;
                D[a * CS_BC_KB + b] = M[(l0 + a) * nc + k0 + b];
            }
            __syncthreads();
            __shared__ int okD;
            if (threadIdx.x < 32) {
                const bool ok = bc_warp_inverse(D, kn);
                if (threadIdx.x == 0) okD = ok ? 1 : 0;
            }
            __syncthreads();
            for (int q = threadIdx.x; q < nc; q += blockDim.x) {
                const int c = q - k0;
                if (!okD || (c >= 0 && c < kn)) {
                    for (int t = 0; t < kn; t++) lbuf[t * nc + q] = okD ? D[t * CS_BC_KB + c] : 0.f;
                    continue;
                }
                bc_block_rows_times(D, M + (size_t)l0 * nc + q, nc, kn, lbuf + q, nc);
            }
            if (threadIdx.x == 0) lbuf[CS_BC_KB * nc] = okD ? 1.f : 0.f;
        }
        cluster.sync();
        if (rank != owner) {
            const float4* ob4 = reinterpret_cast<const float4*>(cluster.map_shared_rank(lbuf, owner));
            float4* lb4 = reinterpret_cast<float4*>(lbuf);
            for (int q = threadIdx.x; q < UB / 4; q += blockDim.x) lb4[q] = ob4[q];
        }
        __syncthreads();
        if (lbuf[CS_BC_KB * nc] == 0.f) {  // the same flag in every CTA: a uniform exit
            if (threadIdx.x == 0) bad = 1;
            break;
        }
        const int ownRow0 = rank == owner ? CS_BC_KB * (kb / CS_BC_CLUSTER) : -CS_BC_KB;  // this CTA's rows of K
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int j = h ? j1 : j0;
            if (j >= nc) continue;
            float uj[CS_BC_KB];
#pragma unroll
            for (int t = 0; t < CS_BC_KB; t++) uj[t] = t < kn ? lbuf[t * nc + j] : 0.f;
            const bool jk = j >= k0 && j < k0 + kn;
            for (int l4 = 0; l4 < R; l4 += 4) {  // RM is a multiple of 12: rows l4..l4+3 exist in colb
                float t[4];
                bc_dot12x4(colb + l4 * CS_BC_KB, uj, t);
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const int li = l4 + r;
                    if (li >= R) break;
                    float v;
                    if (li >= ownRow0 && li < ownRow0 + kn) v = lbuf[(li - ownRow0) * nc + j];
                    else v = jk ? -t[r] : M[li * nc + j] - t[r];
                    M[li * nc + j] = v;
                }
            }
        }
        __syncthreads();
    }
    cluster.sync();
    if (!bad)
        for (int e = threadIdx.x; e < R * nc; e += blockDim.x) {
            const int li = e / nc, j = e - li * nc;
            G[(size_t)grow(li) * nc + j] = M[e];
        }
    __threadfence();
    cluster.sync();
    float* Inv = B.bc_inv + sh.bc_mat_off;
    if (!bad)
        for (int e = threadIdx.x; e < R * nc; e += blockDim.x) {
            const int li = e / nc, j = e - li * nc;
            const int i = grow(li);
            Inv[(size_t)i * nc + j] = 0.5f * (M[e] + __ldcg(&G[(size_t)j * nc + i]));
        }
    if (rank == 0 && threadIdx.x == 0) B.bc_ok[s] = bad ? 0 : 1;
}

// R r: a block per aggregate sums r over its member nodes (thread-strided over the ascending
// members, then a fixed-order block sum) in FP64, stored in FP32.
__global__ void __launch_bounds__(256) cs_bc_restrict_kernel(Batch B) {
    __shared__ double sh3[3 * 8];
    const int w = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (w >= B.bc_total_agg) return;
    const int2 sa = B.bc_agg[w];
    if (!bc_trip_on(B, sa.x)) return;
    const SheetDesc& sh = B.sheets[sa.x];
    const int m0 = B.bc_mptr[sh.bc_agg_off + sa.y], m1 = B.bc_mptr[sh.bc_agg_off + sa.y + 1];
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    for (int m = m0 + (int)threadIdx.x; m < m1; m += blockDim.x) {
        const int node = sh.node_off + B.bc_mem[sh.bc_mem_off + m];
        r0 += (double)B.r[3 * node];
        r1 += (double)B.r[3 * node + 1];
        r2 += (double)B.r[3 * node + 2];
    }
    r0 = bc_warp_sum(r0);
    r1 = bc_warp_sum(r1);
    r2 = bc_warp_sum(r2);
    if (lane == 0) {
        sh3[3 * wid] = r0;
        sh3[3 * wid + 1] = r1;
        sh3[3 * wid + 2] = r2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += sh3[3 * q + threadIdx.x];
        B.bc_rc[sh.bc_vec_off + 3 * sa.y + threadIdx.x] = (float)t;
    }
}

// e_c = A_c^-1 R r: a warp per coarse row (lane-strided columns, then a butterfly).
__global__ void __launch_bounds__(256) cs_bc_apply_kernel(Batch B) {
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= 3 * B.bc_total_agg) return;
    const int2 sa = B.bc_agg[w / 3];
    if (!bc_trip_on(B, sa.x)) return;
    const SheetDesc& sh = B.sheets[sa.x];
    const int nc = 3 * sh.bc_na, i = 3 * sa.y + w % 3;
    const float* row = B.bc_inv + sh.bc_mat_off + (size_t)i * nc;
    const float* rc = B.bc_rc + sh.bc_vec_off;
    float acc = 0.f;
    for (int j = lane; j < nc; j += 32) acc = __fmaf_rn(row[j], rc[j], acc);
    acc = bc_warp_sum(acc);
    if (lane == 0) B.bc_ec[sh.bc_vec_off + i] = acc;
}

// z += R^T e_c over the rows of the slice index's natural-order chunk (as cs_vector_kernel takes
// them), and that chunk's r.z and r.r partials recomputed with the corrected z.
__global__ void __launch_bounds__(128) cs_bc_finish_kernel(Batch B) {
    const int slice = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (slice >= B.n_slices) return;
    const SliceDesc sd = B.slices[slice];
    if (!bc_trip_on(B, sd.sheet)) return;
    const SheetDesc& sh = B.sheets[sd.sheet];
    const bool mixed = B.params->mixed != 0;
    const bool live = lane < sd.rows;
    const int local = CS_SLICE * (slice - sh.slice_off) + lane;
    double rz = 0.0, rr = 0.0;
    float rzf = 0.f, rrf = 0.f;
    if (live) {
        const int row = sh.node_off + local;
        const float* ec = B.bc_ec + sh.bc_vec_off + 3 * B.bc_node_agg[sh.bc_node_off + local];
        float r[3], z[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            r[c] = B.r[3 * row + c];
            z[c] = B.z[3 * row + c] + ec[c];
            B.z[3 * row + c] = z[c];
        }
        if (mixed) {
            rz = (double)r[0] * z[0] + (double)r[1] * z[1] + (double)r[2] * z[2];
            rr = (double)r[0] * r[0] + (double)r[1] * r[1] + (double)r[2] * r[2];
        } else {
            rzf = r[0] * z[0] + r[1] * z[1] + r[2] * z[2];
            rrf = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        }
    }
    if (mixed) {
        rz = bc_warp_sum(rz);
        rr = bc_warp_sum(rr);
    } else {
        rz = (double)bc_warp_sum(rzf);
        rr = (double)bc_warp_sum(rrf);
    }
    if (lane == 0) {
        B.part[2 * slice] = rz;
        B.part[2 * slice + 1] = rr;
    }
}

// ---------------------------------------------------------------------------------------
// Coarse matrix of each resident sheet, for the coarse-space correction of the cluster-resident
// solver (resident.cu): A_c = R A R^T, where R sums the rows of each aggregate (a segment of a
// CTA's strip) per component, so block (a, b) of A_c is the sum of the stored blocks A_ij with
// row i in aggregate a and column j in aggregate b.  The loader lists those blocks per pair
// (a, b) in slot order; a warp sums a pair, lane l taking the blocks l, l + 32, ... in order,
// and a butterfly combines the lanes (a fixed order: deterministic, no atomics).  A_c is SPD (A
// is, and R has full row rank), so Gauss-Jordan elimination inverts it in place in shared memory
// without pivoting, in FP32, with pivot blocks of CS_BC_KB rows.  Per block K (kn rows from k0):
// D = A[K, K] is inverted by one warp (bc_warp_inverse); the rows K become U = D^-1 A[K, :] with
// U[:, K] = D^-1, a thread per column in place; every row i outside K gets A[i, j] -= A[i, K]
// U[:, j] on the columns outside K, and after a barrier A[i, K] = -A[i, K] D^-1 (a thread per
// row).  Five barriers per block.  The inverse, symmetrised, is stored per work item for the
// resident kernel, which applies its CTA's rows each CG iteration.  A non-positive or
// non-finite pivot marks the work item's coarse matrix invalid and the solve runs without the
// correction.  One CTA per resident work item; dynamic shared memory cs_coarse_setup_smem(nc).
namespace {

__device__ __forceinline__ void coarse_load_block(const Batch& B, const SheetDesc& sh, int slot, float (&a)[9]) {
    const float* pk = B.A + (size_t)(sh.panel_off + slot / CS_SLICE) * CS_PANEL_FLOATS;
    const int l = slot % CS_SLICE;
    const float4 a0 = __ldg(reinterpret_cast<const float4*>(pk) + l);
    const float4 a1 = __ldg(reinterpret_cast<const float4*>(pk + 128) + l);
    a[0] = a0.x;
    a[1] = a0.y;
    a[2] = a0.z;
    a[3] = a0.w;
    a[4] = a1.x;
    a[5] = a1.y;
    a[6] = a1.z;
    a[7] = a1.w;
    a[8] = __ldg(pk + 256 + l);
}

}  // namespace

__global__ void __launch_bounds__(CS_COARSE_THREADS) cs_coarse_setup_kernel(Batch B) {
    extern __shared__ __align__(16) float cs_coarse_sm[];
    __shared__ int bad;
    const DevParams& P = *B.params;
    if (P.solver != CS_SOLVER_AUTO_DEV || P.cheb_degree < 3 || !P.coarse) return;  // uniform
    const int idx = blockIdx.x;
    if (idx >= B.n_resident) return;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    const SheetDesc& sh = B.sheets[B.rlist[idx]];
    const int4 ci = B.rcoarse[sh.topo];
    const int nc = ci.x;
    if (nc == 0 || nc > B.res_cnc) {
        if (tid == 0) B.cvalid[idx] = 0;
        return;
    }
    const int ld = cs_coarse_ld(nc);
    float* M = cs_coarse_sm;             // nc x ld
    float* D = M + (size_t)nc * ld;      // CS_BC_KB x CS_BC_KB
    for (int i = tid; i < nc * ld; i += blockDim.x) M[i] = 0.f;
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int q = ci.z + w; q < ci.w; q += nw) {
        const int4 pr = B.cpair[q];
        float acc[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int k = pr.z + lane;
        // two of the lane's blocks in flight at a time, added in order
        for (; k + 32 < pr.w; k += 64) {
            float a0[9], a1[9];
            coarse_load_block(B, sh, __ldg(&B.ccontrib[k]), a0);
            coarse_load_block(B, sh, __ldg(&B.ccontrib[k + 32]), a1);
#pragma unroll
            for (int e = 0; e < 9; e++) acc[e] += a0[e];
#pragma unroll
            for (int e = 0; e < 9; e++) acc[e] += a1[e];
        }
        if (k < pr.w) {
            float a0[9];
            coarse_load_block(B, sh, __ldg(&B.ccontrib[k]), a0);
#pragma unroll
            for (int e = 0; e < 9; e++) acc[e] += a0[e];
        }
#pragma unroll
        for (int e = 0; e < 9; e++) acc[e] = bc_warp_sum(acc[e]);
        if (lane == 0) {
#pragma unroll
            for (int e = 0; e < 9; e++) M[(size_t)(3 * pr.x + e / 3) * ld + 3 * pr.y + e % 3] = acc[e];
        }
    }
    __syncthreads();
    const int rs = blockDim.x / nc;  // rows whose updates run together (nc <= blockDim)
    const int j = tid % nc, i0 = tid / nc;
    for (int k0 = 0; k0 < nc; k0 += CS_BC_KB) {
        const int kn = min(CS_BC_KB, nc - k0);
        for (int e = tid; e < kn * kn; e += blockDim.x) {
            const int a = e / kn, b = e - a * kn;
            D[a * CS_BC_KB + b] = M[(size_t)(k0 + a) * ld + k0 + b];
        }
        __syncthreads();
        if (w == 0) {
            const bool ok = bc_warp_inverse(D, kn);
            if (lane == 0 && !ok) bad = 1;
        }
        __syncthreads();
        if (bad) break;  // uniform: read after the barrier
        // rows K become U = D^-1 A[K, :] (U[:, K] = D^-1), a thread per column, in place
        for (int q = tid; q < nc; q += blockDim.x) {
            float* col = M + (size_t)k0 * ld + q;
            const int c = q - k0;
            if (c >= 0 && c < kn) {
                for (int t = 0; t < kn; t++) col[(size_t)t * ld] = D[t * CS_BC_KB + c];
                continue;
            }
            float av[CS_BC_KB];
#pragma unroll
            for (int v = 0; v < CS_BC_KB; v++) av[v] = v < kn ? col[(size_t)v * ld] : 0.f;
#pragma unroll
            for (int t = 0; t < CS_BC_KB; t++) {
                if (t >= kn) break;
                float x = 0.f, y = 0.f;
#pragma unroll
                for (int v = 0; v < CS_BC_KB; v += 2) {
                    if (v < kn) x = __fmaf_rn(D[t * CS_BC_KB + v], av[v], x);
                    if (v + 1 < kn) y = __fmaf_rn(D[t * CS_BC_KB + v + 1], av[v + 1], y);
                }
                col[(size_t)t * ld] = x + y;
            }
        }
        __syncthreads();
        // rows outside K, columns outside K: A[i, j] -= A[i, K] U[:, j]
        if (i0 < rs && !(j >= k0 && j < k0 + kn)) {
            float uj[CS_BC_KB];
#pragma unroll
            for (int t = 0; t < CS_BC_KB; t++) uj[t] = t < kn ? M[(size_t)(k0 + t) * ld + j] : 0.f;
#pragma unroll 2
            for (int i = i0; i < nc; i += rs) {
                if (i >= k0 && i < k0 + kn) continue;
                const float* ai = M + (size_t)i * ld + k0;  // 16-byte aligned: ld and k0 are multiples of 4
                float x, y;
                if (kn == CS_BC_KB) {
                    const float4* a4 = reinterpret_cast<const float4*>(ai);
                    const float4 a = a4[0], b = a4[1], c = a4[2];
                    x = a.x * uj[0];
                    y = a.y * uj[1];
                    x = __fmaf_rn(a.z, uj[2], x);
                    y = __fmaf_rn(a.w, uj[3], y);
                    x = __fmaf_rn(b.x, uj[4], x);
                    y = __fmaf_rn(b.y, uj[5], y);
                    x = __fmaf_rn(b.z, uj[6], x);
                    y = __fmaf_rn(b.w, uj[7], y);
                    x = __fmaf_rn(c.x, uj[8], x);
                    y = __fmaf_rn(c.y, uj[9], y);
                    x = __fmaf_rn(c.z, uj[10], x);
                    y = __fmaf_rn(c.w, uj[11], y);
                } else {
                    x = 0.f;
                    y = 0.f;
                    for (int t = 0; t < kn; t++) x = __fmaf_rn(ai[t], uj[t], x);
                }
                M[(size_t)i * ld + j] -= x + y;
            }
        }
        __syncthreads();
        // rows outside K, columns K: A[i, K] = -A[i, K] D^-1, a thread per row
        for (int i = tid; i < nc; i += blockDim.x) {
            if (i >= k0 && i < k0 + kn) continue;
            float* ai = M + (size_t)i * ld + k0;
            float av[CS_BC_KB];
#pragma unroll
            for (int v = 0; v < CS_BC_KB; v++) av[v] = v < kn ? ai[v] : 0.f;
#pragma unroll
            for (int c = 0; c < CS_BC_KB; c++) {
                if (c >= kn) break;
                float x = 0.f;
#pragma unroll
                for (int v = 0; v < CS_BC_KB; v++)
                    if (v < kn) x = __fmaf_rn(av[v], D[v * CS_BC_KB + c], x);
                ai[c] = -x;
            }
        }
        __syncthreads();
    }
    // written out symmetrised
    float* out = B.cinv + (size_t)idx * B.res_cnc * B.res_cnc;
    if (!bad)
        for (int i = w; i < nc; i += nw)
            for (int jj = lane; jj < nc; jj += 32) out[(size_t)i * nc + jj] = 0.5f * (M[(size_t)i * ld + jj] + M[(size_t)jj * ld + i]);
    if (tid == 0) B.cvalid[idx] = bad ? 0 : 1;
}
