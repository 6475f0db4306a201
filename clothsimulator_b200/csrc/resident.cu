// Cluster-resident PCG: one thread-block cluster solves one sheet with the sheet's system
// held in the cluster's distributed shared memory for the whole solve.
//
// The batched loop of pcg.cu streams every sheet's matrix from HBM once per CG iteration
// (about 1.7 MB per 64x64 sheet, ~300 iterations per step).  A sheet of that size fits in
// the shared memory of a cluster of 8 to 10 CTAs (227 KB each), so here each cluster
//   * takes the next sheet from a device work counter (persistent clusters; a sheet that
//     converges early frees its cluster at once, there is no batch-wide tail),
//   * copies its share of the sheet's SELL-32 panels (a contiguous strip of slices) into
//     shared memory once per solve,
//   * runs the per-instance state machine of the batched loop (FP32 CG on the correction
//     system, FP64 dot products and norms, FP64 residual replacements with the search
//     direction kept (reliable updates), warm-start guard, inner and outer stopping tests)
//     with the FP32 vectors in registers, one thread per row.  The CG recurrence is the
//     Chronopoulos-Gear form: per iteration one SpMV w = A u and ONE fused reduction of
//     (r.u, w.u, r.r), instead of two reductions;
//   * preconditions with the 3x3 block-Jacobi inverse or, when asked and the sheet's strips
//     keep enough of its couplings, with a Chebyshev polynomial in the block-Jacobi-scaled
//     strip of rows each CTA holds (its SpMVs read only the CTA's own shared memory);
//   * exchanges data without cluster barriers: after u = P^-1 r each CTA pushes the values
//     of its strip's boundary rows into the halo slots of the CTAs that read them with
//     st.async remote stores, which complete bytes on the receiver's mbarrier; reduction
//     partials travel the same way.  A CTA waits only on its own mbarriers.  Sends for step
//     k+1 depend on every CTA's step-k partial, so one halo buffer and two reduction buffers
//     suffice (a sender is never two steps ahead of a receiver);
//   * sums deterministically: a butterfly within each warp (IEEE addition is commutative, so
//     every lane ends with the same bits), then warp and CTA partials in a fixed order, every
//     CTA summing the same partials: all CTAs take identical decisions;
//   * runs the SpMV's local slots while the halo values travel, the halo slots after.
// Every wait is bounded.  A CTA whose wait runs out raises an abort flag in all CTAs and an
// error word for the host, and all CTAs leave through the kernel's final cluster barrier (the
// only one after start-up), so no CTA exits while another may still address its memory.
// Rows of a slice beyond the shared-memory panel budget are read from global memory.
//
// Replaces the reference's per-cloth GPU solve (Cloth.cu:766-809) like pcg.cu does; the
// block-Jacobi preconditioner is the 3x3 block inverse from the gather kernel (the reference
// builds the scalar Jacobi one, PhysicsHelper.cu:479-485).
#include <cooperative_groups.h>

#include "cs_internal.h"

namespace cg = cooperative_groups;

namespace {

constexpr uint32_t RES_WAIT_TRIES = 1u << 22;  // polls of a phase before a CTA gives up (about 0.1 s)
#ifndef RES_POLL_NS
#define RES_POLL_NS 32
#endif

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t mapa(uint32_t a, int rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}

__device__ __forceinline__ void rbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void rbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Non-blocking test of a phase (test_wait, not try_wait: try_wait may suspend the thread for
// a system-defined time).  CLUSTER = false: acquire at CTA scope, enough for data that
// st.async wrote into this CTA's shared memory with completion on this mbarrier; true:
// cluster scope, for the residual signal that orders other CTAs' global-memory writes.
template <bool CLUSTER>
__device__ __forceinline__ bool rbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    if (CLUSTER)
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
    return ok != 0;
}

// Remote arrive on another CTA's mbarrier, releasing this thread's prior writes cluster-wide.
__device__ __forceinline__ void rbar_arrive_remote(uint32_t cbar) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cbar) : "memory");
}

__device__ __forceinline__ void st_async_f4(uint32_t caddr, float4 v, uint32_t cbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(caddr),
                 "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "r"(cbar)
                 : "memory");
}

__device__ __forceinline__ void st_async_d2(uint32_t caddr, double a, double b, uint32_t cbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(caddr), "d"(a),
                 "d"(b), "r"(cbar)
                 : "memory");
}

__device__ __forceinline__ void st_async_u32(uint32_t caddr, uint32_t v, uint32_t cbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(caddr), "r"(v), "r"(cbar)
                 : "memory");
}

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

// Shared control block of one CTA.
struct __align__(16) ResShared {
    double red[2][CS_RES_MAX_CL][4];   // reduction partials by sender rank, two buffers
    double wsum[CS_RES_MAX_WARPS][4];  // warp partials
    uint64_t bar[5];                   // 0 halo, 1-2 reduction buffers, 3 residual signal, 4 work item
    int next;                          // work item sent by rank 0
    int abort_flag;                    // raised by any CTA whose wait ran out
    // strip-local Chebyshev preconditioner of the current sheet: degree (1: block-Jacobi),
    // 1/theta, and per step k the coefficients of d_k = a_k d_{k-1} + b_k P^-1 (r - A_loc x)
    int cheb_deg;
    float cheb_inv_th;
    float cheb_a[CS_PRECOND_MAX_DEGREE], cheb_b[CS_PRECOND_MAX_DEGREE];
};

constexpr float CHEB_LMAX_MARGIN = 1.1f; // the estimate approaches lambda_max from below
constexpr float CHEB_LMIN_RATIO = 1.0f / 30.0f;

// Waits for `parity` of `bar` on every thread, at most RES_WAIT_TRIES polls, giving up early
// once another CTA raised the abort flag.  Returns true on every thread only if the whole
// CTA saw the phase complete.
template <bool CLUSTER = false>
__device__ __forceinline__ bool res_wait(ResShared& S, uint32_t bar, uint32_t parity) {
    bool ok = false;
    for (uint32_t t = 0; t < RES_WAIT_TRIES; t++) {
        if (rbar_test<CLUSTER>(bar, parity)) {
            ok = true;
            break;
        }
        if (*(volatile int*)&S.abort_flag) break;
        // back off: polls share the shared-memory pipe with the remote stores being awaited
        __nanosleep(RES_POLL_NS);
    }
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// Raises the abort flag in every CTA of the cluster and the error word for the host.
__device__ __forceinline__ void res_abort(const cg::cluster_group& cl, ResShared& S, int ncta, int* err) {
    if (threadIdx.x == 0) {
        for (int c = 0; c < ncta; c++) *(volatile int*)cl.map_shared_rank(&S.abort_flag, c) = 1;
        atomicExch(err, 1);
    }
}

// Cluster-wide sum of three values (fp32: in float, the plain FP32 solver; else double).
// Order: a butterfly within each warp, then the warp partials in warp order, then the CTA
// partials in rank order.  The last two are serial sums over broadcast shared-memory reads,
// done redundantly by every thread that needs the result (no shuffles: with ~20 warps per SM
// the shuffle pipe is the bottleneck of a butterfly).  Every CTA sums the same partials in
// the same order, so all threads of the cluster return identical sums.  Partials travel by
// st.async into buffer `nred & 1` of every CTA.  Returns false if the wait gave up (the
// caller aborts).
__device__ __forceinline__ bool cluster_sum3(ResShared& S, int rank, int ncta, uint32_t& nred, double (&v)[3], bool fp32) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int b = (int)(nred & 1u);
#pragma unroll
    for (int i = 0; i < 3; i++) v[i] = fp32 ? (double)rwarp_sum((float)v[i]) : rwarp_sum(v[i]);
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < 3; i++) S.wsum[w][i] = v[i];
    }
    __syncthreads();
    if (w == 0 && lane < ncta) {
        // unrolled to the compile-time bound so every load issues before the add chain
        double t[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (fp32) {
                float a = 0.f;
#pragma unroll
                for (int j = 0; j < CS_RES_MAX_WARPS; j++)
                    if (j < nw) a += (float)S.wsum[j][i];
                t[i] = (double)a;
            } else {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < CS_RES_MAX_WARPS; j++)
                    if (j < nw) a += S.wsum[j][i];
                t[i] = a;
            }
        }
        const uint32_t bar = saddr(&S.bar[1 + b]);
        if (lane == 0) rbar_expect(bar, (uint32_t)ncta * 32u);
        const uint32_t dst = mapa(saddr(&S.red[b][rank][0]), lane);
        const uint32_t dbar = mapa(bar, lane);
        st_async_d2(dst, t[0], t[1], dbar);
        st_async_d2(dst + 16, t[2], 0.0, dbar);
    }
    const bool ok = res_wait(S, saddr(&S.bar[1 + b]), (nred >> 1) & 1u);
    nred++;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (fp32) {
            float a = 0.f;
#pragma unroll
            for (int c = 0; c < CS_RES_MAX_CL; c++)
                if (c < ncta) a += (float)S.red[b][c][i];
            v[i] = (double)a;
        } else {
            double a = 0.0;
#pragma unroll
            for (int c = 0; c < CS_RES_MAX_CL; c++)
                if (c < ncta) a += S.red[b][c][i];
            v[i] = a;
        }
    }
    return ok;
}

// The coarse-space correction's state in one CTA's shared memory: the coarse region the loader
// sizes with coarseSmemBytes, each part rounded up to 4 floats.  Offsets come from the kernel
// parameters (res_cnc = nc, res_ck = K), so they hold no registers.
//   ai   this CTA's rows of the inverse coarse matrix, 3K x nc
//   r32  the coarse residual R r in FP32 (the matrix-vector product's input), nc
//   ce   the correction of this CTA's aggregates, 3K (CP = 3K rounded up to 4)
//   part this CTA's segment sums before they are sent, CP
//   red  every CTA's segment sums: [buffer][rank][CP]
//   r64, s64  the coarse residual R r and search direction R s in FP64, nc each
struct CoarseSm {
    unsigned char* base;
    int nc, k3, cp;
    __device__ __forceinline__ CoarseSm(unsigned char* b, int nc_, int k) : base(b), nc(nc_), k3(3 * k), cp((3 * k + 3) / 4 * 4) {}
    __device__ __forceinline__ static int r4(int n) { return (n + 3) / 4 * 4; }
    __device__ __forceinline__ float* ai() const { return reinterpret_cast<float*>(base); }
    __device__ __forceinline__ float* r32() const { return ai() + r4(k3 * nc); }
    __device__ __forceinline__ float* ce() const { return r32() + r4(nc); }
    __device__ __forceinline__ float* part() const { return ce() + cp; }
    __device__ __forceinline__ float* red() const { return part() + cp; }
    __device__ __forceinline__ double* r64(int ncta) const { return reinterpret_cast<double*>(red() + 2 * ncta * cp); }
    __device__ __forceinline__ double* s64(int ncta) const { return r64(ncta) + nc; }
    // entry q of the coarse vector in one buffer of `red` (rank q / 3K, segment and component
    // q % 3K)
    __device__ __forceinline__ int off(int q) const { return (q / k3) * cp + q % k3; }
};

// cluster_sum3 that also carries the coarse vector R y of a per-row vector y.  The lanes of a
// slice hold the rows of one segment consecutively (the loader orders them so); `cseg` packs this
// lane's run: the run's first lane (bits 0-4), whether this lane ends it (bit 5), the segment + 1
// (bits 8-15; 0 for a lane without a row) and, for the gathering lanes of warp 1, the warps
// holding the lane's segment (bits 16-31); bit 6 is the caller's.  A segmented inclusive scan (5 shuffle steps per
// component) leaves each run's sum in its last lane, which stages it in `wp` (warp-major, CP
// floats per warp); after the first barrier lane 3k + c of warp 1 adds component c of segment
// k over the warps holding it (bits 16-31 of its cseg), in warp order, and those sums travel
// with the three values to every CTA.  On return buffer (nred - 1) & 1 of C.red holds R y, entry
// q at C.off(q) (q = 3 (rank K + k) + c); it may be overwritten by the reduction after next.
// Deterministic like cluster_sum3.
__device__ __forceinline__ bool cluster_sum3c(ResShared& S, int rank, int ncta, uint32_t& nred, double (&v)[3], bool fp32,
                                              const float (&y)[3], bool live, int cseg, float* wp, const CoarseSm& C) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int b = (int)(nred & 1u);
    {
        const int rs = cseg & 31, sg = ((cseg >> 8) & 0xff) - 1;
        float a0 = live ? y[0] : 0.f, a1 = live ? y[1] : 0.f, a2 = live ? y[2] : 0.f;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const float t0 = __shfl_up_sync(0xffffffffu, a0, d), t1 = __shfl_up_sync(0xffffffffu, a1, d),
                        t2 = __shfl_up_sync(0xffffffffu, a2, d);
            if (lane - d >= rs) {
                a0 += t0;
                a1 += t1;
                a2 += t2;
            }
        }
        if (((cseg >> 5) & 1) && sg >= 0 && 3 * sg < C.k3) {
            wp[w * C.cp + 3 * sg] = a0;
            wp[w * C.cp + 3 * sg + 1] = a1;
            wp[w * C.cp + 3 * sg + 2] = a2;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) v[i] = fp32 ? (double)rwarp_sum((float)v[i]) : rwarp_sum(v[i]);
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < 3; i++) S.wsum[w][i] = v[i];
    }
    __syncthreads();
    double t[3] = {0.0, 0.0, 0.0};
    if (w == 0 && lane < ncta) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (fp32) {
                float a = 0.f;
#pragma unroll
                for (int j = 0; j < CS_RES_MAX_WARPS; j++)
                    if (j < nw) a += (float)S.wsum[j][i];
                t[i] = (double)a;
            } else {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < CS_RES_MAX_WARPS; j++)
                    if (j < nw) a += S.wsum[j][i];
                t[i] = a;
            }
        }
    }
    if (w == 1 && lane < C.cp) {
        float a = 0.f;
        const unsigned wk = (unsigned)cseg >> 16;  // the warps holding this lane's segment
#pragma unroll
        for (int j = 0; j < CS_RES_MAX_WARPS; j++)
            if ((wk >> j) & 1u) a += wp[j * C.cp + lane];
        C.part()[lane] = a;
    }
    // warps 0 and 1 only (named barrier 1 of 64 threads): the segment sums are in place before
    // warp 0 sends them; the other warps go straight to the wait
    if (w < 2) asm volatile("bar.sync 1, 64;" ::: "memory");
    if (w == 0 && lane < ncta) {
        const uint32_t bar = saddr(&S.bar[1 + b]);
        if (lane == 0) rbar_expect(bar, (uint32_t)ncta * (32u + 4u * (uint32_t)C.cp));
        const uint32_t dst = mapa(saddr(&S.red[b][rank][0]), lane);
        const uint32_t dbar = mapa(bar, lane);
        st_async_d2(dst, t[0], t[1], dbar);
        st_async_d2(dst + 16, t[2], 0.0, dbar);
        const uint32_t cdst = mapa(saddr(C.red() + ((size_t)b * ncta + rank) * C.cp), lane);
        for (int q = 0; q < C.cp / 4; q++) st_async_f4(cdst + 16u * q, reinterpret_cast<const float4*>(C.part())[q], dbar);
    }
    const bool ok = res_wait(S, saddr(&S.bar[1 + b]), (nred >> 1) & 1u);
    nred++;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (fp32) {
            float a = 0.f;
#pragma unroll
            for (int c = 0; c < CS_RES_MAX_CL; c++)
                if (c < ncta) a += (float)S.red[b][c][i];
            v[i] = (double)a;
        } else {
            double a = 0.0;
#pragma unroll
            for (int c = 0; c < CS_RES_MAX_CL; c++)
                if (c < ncta) a += S.red[b][c][i];
            v[i] = a;
        }
    }
    return ok;
}

// CTA-wide sums of two values in FP64, in a fixed order (warp butterfly, then warp partials in
// warp order); every thread returns the same sums.  Ends with a barrier, so S.wsum is free again.
__device__ __forceinline__ void cta_sum2(ResShared& S, double& a, double& b) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    a = rwarp_sum(a);
    b = rwarp_sum(b);
    if (lane == 0) {
        S.wsum[w][0] = a;
        S.wsum[w][1] = b;
    }
    __syncthreads();
    double sa = 0.0, sb = 0.0;
    for (int j = 0; j < nw; j++) {
        sa += S.wsum[j][0];
        sb += S.wsum[j][1];
    }
    a = sa;
    b = sb;
    __syncthreads();
}

__device__ __forceinline__ void mat3_vec(const float (&M)[9], const float (&x)[3], float (&y)[3]) {
    y[0] = M[0] * x[0] + M[1] * x[1] + M[2] * x[2];
    y[1] = M[3] * x[0] + M[4] * x[1] + M[5] * x[2];
    y[2] = M[6] * x[0] + M[7] * x[1] + M[8] * x[2];
}

// w += (row of A) u over the row's block slots whose u entry is local (HALO = false: own
// rows) or a halo copy (HALO = true), fully unrolled so that every slot's panel and u loads
// are in flight together.  The local pass runs while the halo values travel.  `cw` holds the
// slots' indices into this CTA's u array (own rows below `halo0`, then the halo slots), two
// 16-bit indices per word.  `pn` points at the row's first panel, in shared memory or
// (beyond the shared-memory budget) in global memory.
template <bool HALO>
__device__ __forceinline__ void row_times_u(const float* __restrict__ pn, int width, const uint32_t (&cw)[CS_RES_MAX_WIDTH / 2],
                                            const float4* su, int halo0, int lane, float& q0, float& q1, float& q2) {
#pragma unroll
    for (int k = 0; k < CS_RES_MAX_WIDTH; k++) {
        const int idx = (int)((cw[k >> 1] >> ((k & 1) * 16)) & 0xffffu);
        if (k < width && (idx >= halo0) == HALO) {
            const float* pk = pn + k * CS_PANEL_FLOATS;
            const float4 a0 = reinterpret_cast<const float4*>(pk)[lane];
            const float4 a1 = reinterpret_cast<const float4*>(pk + 128)[lane];
            const float a8 = pk[256 + lane];
            const float4 pv = su[idx];
            q0 += a0.x * pv.x + a0.y * pv.y + a0.z * pv.z;
            q1 += a0.w * pv.x + a1.x * pv.y + a1.y * pv.z;
            q2 += a1.z * pv.x + a1.w * pv.y + a8 * pv.z;
        }
    }
}

}  // namespace

extern __shared__ __align__(16) unsigned char cs_res_smem[];

// Launch: cluster dimension (CL, 1, 1), blockDim = 32 x (slices per CTA, at most
// CS_RES_MAX_WARPS), dynamic shared memory = res_cap panels + the u array (res_halo0 own row
// slots, then the halo slots).  Grid: whole clusters, persistent (each takes sheets until
// none is left).  B.loop[5] is the work counter (zeroed by the solve setup), B.loop[6] the
// error word (set when a wait ran out).
__global__ void __launch_bounds__(CS_RES_MAX_WARPS * 32, 1) cs_resident_pcg_kernel(Batch B) {
    const DevParams P = *B.params;
    if (P.solver != CS_SOLVER_AUTO_DEV || B.n_resident == 0) return;  // uniform over the grid
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int ncta = (int)cl.num_blocks();
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    const int cap = B.res_cap, halo0 = B.res_halo0;
    const float* sm_panels = reinterpret_cast<const float*>(cs_res_smem);
    float4* su = reinterpret_cast<float4*>(cs_res_smem + (size_t)cap * CS_PANEL_FLOATS * sizeof(float));
    __shared__ ResShared S;
    if (tid == 0) {
        rbar_init(saddr(&S.bar[0]), 1);
        rbar_init(saddr(&S.bar[1]), 1);
        rbar_init(saddr(&S.bar[2]), 1);
        rbar_init(saddr(&S.bar[3]), (uint32_t)ncta);
        rbar_init(saddr(&S.bar[4]), 1);
        S.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cl.sync();  // every CTA's barriers exist before any remote arrive or st.async
    const uint32_t hbar = saddr(&S.bar[0]), sbar = saddr(&S.bar[3]), ibar = saddr(&S.bar[4]);
    uint32_t nhalo = 0, nred = 0, nres = 0, nitem = 0;
    const bool mixed = P.mixed != 0, fp32 = !mixed;
    const int myslot = w * CS_SLICE + lane;
    int* err = B.loop + 6;

    for (;;) {
        // work item: rank 0 takes the next sheet and sends its index to every CTA
        if (tid == 0) rbar_expect(ibar, 4u);
        if (rank == 0 && tid == 0) {
            const int nx = atomicAdd(&B.loop[5], 1);
            for (int c = 0; c < ncta; c++) st_async_u32(mapa(saddr(&S.next), c), (uint32_t)nx, mapa(ibar, c));
        }
        if (!res_wait(S, ibar, nitem & 1u)) {
            res_abort(cl, S, ncta, err);
            break;
        }
        nitem++;
        const int idx = S.next;
        if (idx >= B.n_resident) break;

        const int s = B.rlist[idx];
        const SheetDesc sh = B.sheets[s];
        const int tb = sh.topo * (CS_RES_MAX_CL + 1);
        const int lo = B.rsplit[tb + rank], hi = B.rsplit[tb + rank + 1];
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
            for (int i = tid; i < ncopy; i += blockDim.x) dst[i] = __ldg(src + i);
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
        const int g = sh.node_off + row;
        // u-array indices of the row's slots, packed 16-bit, for the whole solve
        uint32_t cw[CS_RES_MAX_WIDTH / 2];
#pragma unroll
        for (int j = 0; j < CS_RES_MAX_WIDTH / 2; j++) {
            uint32_t lo16 = 0, hi16 = 0;
            if (2 * j < width) lo16 = (uint32_t)__ldg(&B.rcode[(tp + 2 * j) * CS_SLICE + lane]) & 0xfffu;
            if (2 * j + 1 < width) hi16 = (uint32_t)__ldg(&B.rcode[(tp + 2 * j + 1) * CS_SLICE + lane]) & 0xfffu;
            cw[j] = lo16 | (hi16 << 16);
        }
        // halo sends of this CTA (the first one per thread in a register) and bytes it receives
        const int snd0 = B.rsendptr[tb + rank], snd1 = B.rsendptr[tb + rank + 1];
        const uint32_t my_send = snd0 + tid < snd1 ? __ldg(&B.rsend[snd0 + tid]) : 0u;
        const uint32_t halo_bytes = (uint32_t)B.rhalo[tb + rank] * 16u;

        // coarse-space correction (uniform over the cluster): its shared-memory region, this
        // CTA's rows of the inverse coarse matrix, this thread's segment and, for the lanes of
        // warp 1 that sum segments, their slot ranges
        const int4 cinfo = B.rcoarse[sh.topo];
        const bool coarse = P.coarse && P.cheb_degree >= 3 && B.rcheb[tb + rank] && cinfo.x == B.res_cnc &&
                            cinfo.x > 0 && B.cvalid[idx] && nw >= 2;
#define C CoarseSm(cs_res_smem + B.res_coff, B.res_cnc, B.res_ck)
        // the segment masks of this CTA's warps (tb = topology x (CS_RES_MAX_CL + 1))
#define WMASKS (B.rwmask + (tb / (CS_RES_MAX_CL + 1)) * CS_RES_MAX_CL * CS_RES_MAX_WARPS + rank * CS_RES_MAX_WARPS)
        int cseg = 0;  // this lane's segment run, the warps holding its segment (cluster_sum3c)
        // this thread's entry of the coarse vectors in a buffer of C.red (q = tid, the common case)
        const int coff = coarse && tid < C.nc ? C.off(tid) : 0;
        if (coarse) {
            const float* src = B.cinv + (size_t)idx * B.res_cnc * B.res_cnc + (size_t)rank * C.k3 * C.nc;
            for (int i = tid; i < C.k3 * C.nc; i += blockDim.x) C.ai()[i] = __ldcg(src + i);
            for (int i = tid; i < C.nc; i += blockDim.x) C.s64(ncta)[i] = 0.0;
            const int myseg = live ? B.ragg[sh.row2slot_off + row] - rank * B.res_ck : -1;
            // this lane's run of equal segments (consecutive lanes; -1: no row)
            const unsigned same = __match_any_sync(0xffffffffu, myseg);
            cseg = (__ffs(same) - 1) | ((lane == 31 || !((same >> (lane + 1)) & 1u)) ? 32 : 0) |
                   ((live ? myseg + 1 : 0) << 8);
            if (w == 1 && lane < C.k3) {
                // the warps whose rows include this lane's segment (the gather of cluster_sum3c)
                int wk = 0;
                for (int j = 0; j < nw; j++) wk |= ((__ldg(&WMASKS[j]) >> (lane / 3)) & 1) << j;
                cseg |= wk << 16;
            }
        }
        // bit 6 of cseg: the buffer of C.red holding the last coarse vector received

        float Pi[9];
        float e[3] = {0.f, 0.f, 0.f}, r[3] = {0.f, 0.f, 0.f}, u[3], wv[3], p[3] = {0.f, 0.f, 0.f},
              sv3[3] = {0.f, 0.f, 0.f};
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
        double gam = 0.0, gam_prev = 0.0, rr = 0.0, delta = 0.0, alpha_d = 0.0, res0 = bn, resnorm = -1.0,
               first_res = -1.0;
        bool cont = false;  // the next PH_INIT keeps the search direction (reliable update)
        // dv64 and e are known to be zero (zero guess before its first CG step, or a rejected
        // warm start just cleared): the next FP64 residual is b itself and needs no SpMV
        bool dv_zero = !P.warm;
        // the warm start was just scaled by affine_a: the next residual is the affine combination
        // (1 - a) b + a r of b and the residual r of the unscaled start, no SpMV either
        bool affine = false;
        double affine_a = 0.0;
        // the warm start's scaling pass (warm_scale): its first residual gives d.b and d.r
        bool scale_pass = P.warm && P.warm_scale;
        // 1 / gam and 1 / (gam alpha), computed when gam and alpha are set, so that the next
        // iteration's step length costs one division after the reduction instead of three
        double inv_gam = 0.0, inv_ga = 0.0;
        float alpha = 0.f, beta = 0.f;
        int iters = 0, sweeps = 0, sweep_iters = 0, flags = 0, trips = 0;
        // with the coarse correction every solve starts with an FP64 residual: its reduction
        // carries the coarse residual R r that the first preconditioner application needs
        int phase = (P.warm || coarse) ? PH_RES : PH_INIT;
        bool ok = true;

        // q = A_loc x over this CTA's own rows (the strip's diagonal block of A), x in `buf`
        float4* const su_alt = su + B.res_alt;
        auto local_spmv = [&](const float4* buf, float (&q)[3]) {
            q[0] = q[1] = q[2] = 0.f;
            if (in_smem)
                row_times_u<false>(sm_panels + (size_t)lp * CS_PANEL_FLOATS, width, cw, buf, halo0, lane, q[0], q[1], q[2]);
            else
                row_times_u<false>(B.A + (size_t)gp * CS_PANEL_FLOATS, width, cw, buf, halo0, lane, q[0], q[1], q[2]);
        };
        // ce = this CTA's rows of A_c^-1 times the coarse residual (a warp per row, lanes over
        // the columns, butterfly sum: a fixed order)
        auto coarse_matvec = [&]() {
            const float* ai = C.ai();
            const float* r32 = C.r32();
            // rows j and j + nw together (their loads in flight at once), columns fully unrolled
            for (int j = w; j < C.k3; j += 2 * nw) {
                const int j1 = j + nw;
                float a0 = 0.f, a1 = 0.f;
#pragma unroll
                for (int n = 0; n < 6; n++) {
                    const int t = lane + 32 * n;
                    if (t < C.nc) {
                        const float rt = r32[t];
                        a0 = fmaf(ai[j * C.nc + t], rt, a0);
                        if (j1 < C.k3) a1 = fmaf(ai[j1 * C.nc + t], rt, a1);
                    }
                }
                a0 = rwarp_sum(a0);
                if (lane == 0) C.ce()[j] = a0;
                if (j1 < C.k3) {
                    a1 = rwarp_sum(a1);
                    if (lane == 0) C.ce()[j1] = a1;
                }
            }
        };
        // The coarse images of the CG recurrences, replicated in every CTA: with s = w + beta s
        // and the next iteration's r -= alpha s, R s = R w + beta R s and R r -= alpha R s
        // (R w from the reduction just done); R r is what the next preconditioner application
        // reads.  An FP64 residual replaces R r exactly (PH_RES).
        auto coarse_step = [&](double beta_c, double alpha_c) {
            double* s64 = C.s64(ncta);
            double* r64 = C.r64(ncta);
            const float* red = C.red() + (size_t)((cseg >> 6) & 1) * ncta * C.cp;  // R w of the last CG reduction
            for (int q = tid; q < C.nc; q += blockDim.x) {
                const double sq = (double)red[q == tid ? coff : C.off(q)] + beta_c * s64[q];
                s64[q] = sq;
                const double rq = r64[q] - alpha_c * sq;
                r64[q] = rq;
                C.r32()[q] = (float)rq;
            }
        };
        // Strip-local Chebyshev preconditioner: the largest eigenvalue of P^-1 A_loc by power
        // iteration from a hashed +-1 vector (the first barrier also covers the panel copy),
        // then the coefficients of the Chebyshev iteration on [lmax / 30, lmax].  An odd
        // degree keeps the polynomial positive on all of (0, inf), so the preconditioner is
        // SPD whatever the estimate.
        if (P.cheb_degree >= 3 && B.rcheb[tb + rank]) {
            float v[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const uint32_t h = (uint32_t)(3 * row + c) * 0x9E3779B1u;
                v[c] = live ? (((h >> 16) & 1u) ? 1.f : -1.f) : 0.f;
            }
            double lam = 0.0;
            for (int it = 0; it < CS_CHEB_POWER_ITERS; it++) {
                if (live) su_alt[myslot] = make_float4(v[0], v[1], v[2], 0.f);
                __syncthreads();
                float q[3], z[3];
                local_spmv(su_alt, q);
                mat3_vec(Pi, q, z);
                double zz = (double)z[0] * z[0] + (double)z[1] * z[1] + (double)z[2] * z[2];
                double vv = (double)v[0] * v[0] + (double)v[1] * v[1] + (double)v[2] * v[2];
                cta_sum2(S, zz, vv);
                lam = vv > 0.0 ? sqrt(zz / vv) : 0.0;
                const float sc = zz > 0.0 ? (float)(1.0 / sqrt(zz)) : 0.f;
#pragma unroll
                for (int c = 0; c < 3; c++) v[c] = z[c] * sc;
            }
            if (tid == 0) {
                int deg = P.cheb_degree;
                if (!(lam > 0.0) || !rfinite(lam)) deg = 1;
                const float lmax = CHEB_LMAX_MARGIN * (float)lam, lmin = lmax * CHEB_LMIN_RATIO;
                const float th = 0.5f * (lmax + lmin), de = 0.5f * (lmax - lmin), sig = th / de;
                float rho = 1.f / sig;
                S.cheb_inv_th = 1.f / th;
                for (int k = 1; k < deg; k++) {
                    const float rn = 1.f / (2.f * sig - rho);
                    S.cheb_a[k] = rn * rho;
                    S.cheb_b[k] = 2.f * rn / de;
                    rho = rn;
                }
                S.cheb_deg = deg;
            }
        } else if (tid == 0) {
            S.cheb_deg = 1;
        }
        __syncthreads();
        const int cdeg = S.cheb_deg;

        while (phase != PH_FINISH) {
            if (++trips > P.loop_cap) {
                flags |= CS_IF_CAPPED;
                break;
            }
            if (phase == PH_RES) {
                // fold the FP32 correction into the FP64 solution; every CTA signals that its
                // rows are written; then r = b - A dv64 in FP64 over global dv64 (r = b when
                // dv64 is known to be zero: no signal, no SpMV; the decision is uniform)
                const bool zero = dv_zero, aff = affine;
                dv_zero = false;
                affine = false;
                if (live) {
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        B.dv64[3 * g + c] += (double)e[c];
                        e[c] = 0.f;
                    }
                }
                if (!zero && !aff) {
                    __syncthreads();
                    if (tid == 0) {
                        asm volatile("fence.acq_rel.cluster;" ::: "memory");
                        for (int c = 0; c < ncta; c++) rbar_arrive_remote(mapa(sbar, c));
                    }
                    ok = res_wait<true>(S, sbar, nres & 1u);
                    nres++;
                    if (!ok) break;
                }
                double v[3] = {0.0, 0.0, 0.0};
                if (live) {
                    const float* pn = in_smem ? sm_panels + (size_t)lp * CS_PANEL_FLOATS : B.A + (size_t)gp * CS_PANEL_FLOATS;
                    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
                    // four slots' column and dv64 loads in flight at a time; sums in slot order
#pragma unroll
                    for (int k0 = 0; k0 < CS_RES_MAX_WIDTH; k0 += 4) {
                        if (zero || aff || k0 >= width) break;
                        int col[4];
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            col[j] = k0 + j < width ? __ldg(&B.tcol[(tp + k0 + j) * CS_SLICE + lane]) + sh.node_off : g;
                        double d[4][3];
#pragma unroll
                        for (int j = 0; j < 4; j++)
#pragma unroll
                            for (int c = 0; c < 3; c++) d[j][c] = __ldcg(&B.dv64[3 * col[j] + c]);
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            if (k0 + j >= width) break;
                            const float* pk = pn + (size_t)(k0 + j) * CS_PANEL_FLOATS;
                            const float4 a0 = reinterpret_cast<const float4*>(pk)[lane];
                            const float4 a1 = reinterpret_cast<const float4*>(pk + 128)[lane];
                            const float a8 = pk[256 + lane];
                            y0 += (double)a0.x * d[j][0] + (double)a0.y * d[j][1] + (double)a0.z * d[j][2];
                            y1 += (double)a0.w * d[j][0] + (double)a1.x * d[j][1] + (double)a1.y * d[j][2];
                            y2 += (double)a1.z * d[j][0] + (double)a1.w * d[j][1] + (double)a8 * d[j][2];
                        }
                    }
                    double r0 = (double)B.b[3 * g] - y0, r1 = (double)B.b[3 * g + 1] - y1, r2 = (double)B.b[3 * g + 2] - y2;
                    if (aff) {
                        r0 = (1.0 - affine_a) * (double)B.b[3 * g] + affine_a * (double)r[0];
                        r1 = (1.0 - affine_a) * (double)B.b[3 * g + 1] + affine_a * (double)r[1];
                        r2 = (1.0 - affine_a) * (double)B.b[3 * g + 2] + affine_a * (double)r[2];
                    }
                    // drift of the recursive residual it replaces
                    const double q0 = r0 - (double)r[0], q1 = r1 - (double)r[1], q2 = r2 - (double)r[2];
                    r[0] = (float)r0;
                    r[1] = (float)r1;
                    r[2] = (float)r2;
                    if (scale_pass) {
                        const double d0 = B.dv64[3 * g], d1 = B.dv64[3 * g + 1], d2 = B.dv64[3 * g + 2];
                        v[0] = d0 * (double)B.b[3 * g] + d1 * (double)B.b[3 * g + 1] + d2 * (double)B.b[3 * g + 2];
                        v[1] = d0 * r0 + d1 * r1 + d2 * r2;
                    } else {
                        v[0] = r0 * r0 + r1 * r1 + r2 * r2;
                        v[1] = q0 * q0 + q1 * q1 + q2 * q2;
                    }
                }
                if (coarse) {
                    // the coarse residual R r of the replaced r travels with the norms
                    ok = cluster_sum3c(S, rank, ncta, nred, v, false, r, live, cseg, reinterpret_cast<float*>(su_alt), C);
                    const float* red = C.red() + (size_t)((nred - 1) & 1u) * ncta * C.cp;
                    for (int q = tid; q < C.nc; q += blockDim.x) {
                        const float rq = red[q == tid ? coff : C.off(q)];
                        C.r64(ncta)[q] = (double)rq;
                        C.r32()[q] = rq;
                    }
                } else {
                    ok = cluster_sum3(S, rank, ncta, nred, v, false);
                }
                if (!ok) break;
                if (scale_pass) {
                    // d becomes alpha d, alpha = d.b / d.A d (d.A d = d.b - d.r): the multiple of d
                    // nearest to the solution in the energy norm; the next residual is its guard's.
                    // Every CTA holds the same sums, so all take the same branch; each scales its
                    // own rows once every CTA's reads of them are done (they precede the sums).
                    scale_pass = false;
                    const double dad = v[0] - v[1], a = v[0] / dad;
                    if (dad > 0.0 && rfinite(a)) {
                        if (live) {
#pragma unroll
                            for (int c = 0; c < 3; c++) B.dv64[3 * g + c] *= a;
                        }
                        affine = true;  // b - A (a d) = (1 - a) b + a (b - A d)
                        affine_a = a;
                        continue;       // phase stays PH_RES
                    }
                    flags |= CS_IF_WARM_REJECTED;
                    sweeps = 1;
                    res0 = bn;
                    phase = PH_INIT;
                    if (coarse) {
                        if (live) {
#pragma unroll
                            for (int c = 0; c < 3; c++) B.dv64[3 * g + c] = 0.0;
                        }
                        dv_zero = true;
                        phase = PH_RES;
                    }
                    continue;
                }
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
                        if (coarse) {
                            // r = b and its coarse residual come from one more residual of dv = 0
                            if (live) {
#pragma unroll
                                for (int c = 0; c < 3; c++) B.dv64[3 * g + c] = 0.0;
                            }
                            dv_zero = true;
                            phase = PH_RES;
                        }
                        continue;
                    }
                }
                if (aff && (res <= P.tol * bn || bn == 0.0 || iters >= P.max_iters)) {
                    // the solve would end on the affine residual (built from an FP32 copy of r):
                    // an FP64 residual of the scaled start decides instead, so the residual a
                    // finished sheet reports is always an FP64 one
                    phase = PH_RES;
                } else if (res <= P.tol * bn || bn == 0.0) {
                    flags |= CS_IF_CONVERGED;
                    phase = PH_FINISH;
                } else if (iters >= P.max_iters) {
                    flags |= CS_IF_CAPPED;
                    phase = PH_FINISH;
                } else if (mixed || gam == 0.0) {
                    // mixed: a reliable update (the FP64 residual replaced r; the direction
                    // of the last sweep is kept if it ran and r had drifted little); plain:
                    // the first sweep after a warm start
                    res0 = res;
                    cont = mixed && sweep_iters > 0 && !(flags & CS_IF_BREAKDOWN) && sqrt(v[1]) <= CS_RELIABLE_DRIFT * res;
                    phase = PH_INIT;
                } else {
                    // plain FP32 CG stopped on its recursive residual and the FP64 check failed
                    flags |= CS_IF_CAPPED;
                    phase = PH_FINISH;
                }
                continue;
            }
            // PH_INIT (start of a sweep) or PH_CG: u = P^-1 r, halo exchange, w = A u, and
            // one reduction of (r.u, w.u, r.r)
            if (phase == PH_INIT && (flags & CS_IF_WARM_REJECTED) && sweeps == 1 && live) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    B.dv64[3 * g + c] = 0.0;
                    r[c] = B.b[3 * g + c];
                }
            }
            if (phase == PH_CG) {
                dv_zero = false;  // e (folded into dv64 by the next residual) leaves zero here
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    e[c] = __fmaf_rn(alpha, p[c], e[c]);
                    r[c] = __fmaf_rn(-alpha, sv3[c], r[c]);
                }
            }
            mat3_vec(Pi, r, u);
            if (cdeg >= 3) {
                // u = x after cdeg steps of the Chebyshev iteration for A_loc x = r from x = 0.
                // Steps alternate between the two own-row buffers, ending on su_alt (cdeg - 1
                // is even), so one barrier per step orders every write after the reads of the
                // buffer's previous contents, the final su write included.
                float d[3];
                const float ith = S.cheb_inv_th;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    d[c] = u[c] * ith;
                    u[c] = d[c];
                }
                for (int k = 1; k < cdeg; k++) {
                    float4* const buf = (k & 1) ? su : su_alt;
                    if (live) buf[myslot] = make_float4(u[0], u[1], u[2], 0.f);
                    __syncthreads();
                    // the coarse correction of this CTA's aggregates, read after the next barrier
                    if (coarse && k == 1) coarse_matvec();
                    float q[3], t[3];
                    local_spmv(buf, q);
#pragma unroll
                    for (int c = 0; c < 3; c++) q[c] = r[c] - q[c];
                    mat3_vec(Pi, q, t);
                    const float ca = S.cheb_a[k], cb = S.cheb_b[k];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        d[c] = ca * d[c] + cb * t[c];
                        u[c] += d[c];
                    }
                }
            }
            if (coarse) {
                if (cdeg < 3) {
                    // this CTA's spectrum bound failed (block-Jacobi): barriers of its own
                    __syncthreads();
                    coarse_matvec();
                    __syncthreads();
                }
                // u = C r + R^T A_c^-1 R r: the additive coarse-space correction
                if (live) {
#pragma unroll
                    for (int c = 0; c < 3; c++) u[c] += C.ce()[3 * (((cseg >> 8) & 0xff) - 1) + c];
                }
            }
            if (live) su[myslot] = make_float4(u[0], u[1], u[2], 0.f);
            __syncthreads();
            if (tid == 0) rbar_expect(hbar, halo_bytes);
            for (int i = snd0 + tid; i < snd1; i += blockDim.x) {
                const uint32_t m = i == snd0 + tid ? my_send : __ldg(&B.rsend[i]);
                const int d = (int)((m >> 12) & 0xfu);
                st_async_f4(mapa(saddr(&su[halo0 + (int)(m >> 16)]), d), su[m & 0xfffu], mapa(hbar, d));
            }
            wv[0] = wv[1] = wv[2] = 0.f;
            const float* pn = in_smem ? sm_panels + (size_t)lp * CS_PANEL_FLOATS : B.A + (size_t)gp * CS_PANEL_FLOATS;
            if (in_smem)
                row_times_u<false>(sm_panels + (size_t)lp * CS_PANEL_FLOATS, width, cw, su, halo0, lane, wv[0], wv[1], wv[2]);
            else
                row_times_u<false>(pn, width, cw, su, halo0, lane, wv[0], wv[1], wv[2]);
            ok = res_wait(S, hbar, nhalo & 1u);
            nhalo++;
            if (!ok) break;
            if (in_smem)
                row_times_u<true>(sm_panels + (size_t)lp * CS_PANEL_FLOATS, width, cw, su, halo0, lane, wv[0], wv[1], wv[2]);
            else
                row_times_u<true>(pn, width, cw, su, halo0, lane, wv[0], wv[1], wv[2]);
            double v[3] = {0.0, 0.0, 0.0};
            if (live) {
                if (mixed) {
                    v[0] = (double)r[0] * u[0] + (double)r[1] * u[1] + (double)r[2] * u[2];
                    v[1] = (double)wv[0] * u[0] + (double)wv[1] * u[1] + (double)wv[2] * u[2];
                    v[2] = (double)r[0] * r[0] + (double)r[1] * r[1] + (double)r[2] * r[2];
                } else {
                    v[0] = (double)(r[0] * u[0] + r[1] * u[1] + r[2] * u[2]);
                    v[1] = (double)(wv[0] * u[0] + wv[1] * u[1] + wv[2] * u[2]);
                    v[2] = (double)(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                }
            }
            if (coarse) {
                // R w travels with the dot products (the coarse recurrences below)
                ok = cluster_sum3c(S, rank, ncta, nred, v, fp32, wv, live, cseg, reinterpret_cast<float*>(su_alt), C);
                cseg = (cseg & ~64) | (int)(((nred - 1) & 1u) << 6);
            } else {
                ok = cluster_sum3(S, rank, ncta, nred, v, fp32);
            }
            if (!ok) break;
            const double gnew = v[0], dnew = v[1];
            rr = v[2];
            if (phase == PH_INIT && cont) {
                // p = u + beta p and s = w + beta s with beta = (r.u) / (the last iteration's
                // r.u); r no longer follows the recursion that the Chronopoulos-Gear step
                // length assumes, so alpha = r.u / p.s is computed with one more reduction
                cont = false;
                const double bd = gnew / gam_prev;
                if (gnew > 0.0 && rfinite(gnew) && rfinite(bd)) {
                    const float bc = (float)bd;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        p[c] = __fmaf_rn(bc, p[c], u[c]);
                        sv3[c] = __fmaf_rn(bc, sv3[c], wv[c]);
                    }
                    double v2[3] = {0.0, 0.0, 0.0};
                    if (live) v2[0] = (double)p[0] * sv3[0] + (double)p[1] * sv3[1] + (double)p[2] * sv3[2];
                    ok = cluster_sum3(S, rank, ncta, nred, v2, false);
                    if (!ok) break;
                    if (v2[0] > 0.0 && rfinite(v2[0]) && rfinite(gnew / v2[0])) {
                        gam = gnew;
                        delta = dnew;
                        sweep_iters = 0;
                        beta = bc;
                        alpha_d = gnew / v2[0];
                        alpha = (float)alpha_d;
                        inv_gam = 1.0 / gam;
                        inv_ga = 1.0 / (gam * alpha_d);
                        if (coarse) coarse_step((double)bc, alpha_d);
                        phase = PH_CG;
                        continue;
                    }
                }
                // otherwise: restart from p = u below
            }
            if (phase == PH_INIT) {
                gam = gnew;
                delta = dnew;
                sweep_iters = 0;
                beta = 0.f;
                if (!(gam > 0.0 && rfinite(gam))) {
                    phase = PH_RES;
                    continue;
                }
                if (mixed) {
                    alpha_d = gam / delta;
                    alpha = (float)alpha_d;
                    inv_gam = 1.0 / gam;
                    inv_ga = 1.0 / (gam * alpha_d);
                } else {
                    alpha = (float)gam / (float)delta;
                    alpha_d = (double)alpha;
                }
                if (!(delta > 0.0) || !rfinite((double)alpha)) {
                    flags |= CS_IF_BREAKDOWN;
                    phase = PH_RES;
                    continue;
                }
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    p[c] = u[c];
                    sv3[c] = wv[c];
                }
                if (coarse) coarse_step(0.0, alpha_d);
                phase = PH_CG;
                continue;
            }
            // PH_CG: the iteration's x and r updates are done; stopping test on ||r||
            iters += 1;
            sweep_iters += 1;
            // ||r|| against the thresholds, squared (no square root on the critical path)
            bool stop;
            if (mixed) {
                const double ti = P.inner_tol * res0, tt = 0.5 * P.tol * bn;
                stop = rr <= ti * ti || rr <= tt * tt || sweep_iters >= P.sweep_cap;
            } else {
                const double tt = P.tol * bn;
                stop = rr <= tt * tt;
            }
            float nb, na;
            double na_d;
            if (mixed) {
                // beta = gnew / gam; alpha = gnew / (dnew - beta gnew / alpha_prev)
                const double bd = gnew * inv_gam;
                na_d = gnew / (dnew - gnew * gnew * inv_ga);
                nb = (float)bd;
                na = (float)na_d;
            } else {
                nb = (float)gnew / (float)gam;
                na = (float)gnew / ((float)dnew - nb * (float)gnew / alpha);
                na_d = (double)na;
            }
            if (!rfinite((double)nb) || !rfinite((double)na) || !(gnew > 0.0) || !(na > 0.f)) {
                flags |= CS_IF_BREAKDOWN;
                stop = true;
            }
            gam_prev = gam;
            gam = gnew;
            delta = dnew;
            if (stop || iters >= P.max_iters) {
                phase = PH_RES;
                continue;
            }
            beta = nb;
            alpha = na;
            alpha_d = na_d;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                p[c] = __fmaf_rn(beta, p[c], u[c]);
                sv3[c] = __fmaf_rn(beta, sv3[c], wv[c]);
            }
            if (coarse) coarse_step((double)beta, alpha_d);
            if (mixed) {
                inv_gam = 1.0 / gam;
                inv_ga = 1.0 / (gam * alpha_d);
            }
        }
        if (!ok) {
            res_abort(cl, S, ncta, err);
            flags |= CS_IF_BREAKDOWN;
        }
        if (live && (!ok || trips > P.loop_cap)) {
#pragma unroll
            for (int c = 0; c < 3; c++) B.dv64[3 * g + c] += (double)e[c];
        }
        if (rank == 0 && tid == 0) {
            InstState& I = B.inst[s];
            I.rz = gam;
            I.rr = rr;
            I.pq = delta;
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
        if (!ok) break;
    }
#undef C
#undef WMASKS
    cl.sync();  // no CTA leaves while another may still address its shared memory
}
