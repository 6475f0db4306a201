// Learned warm start: a one-ring message-passing MLP that predicts the step's dv, with its
// layers on tcgen05 tensor cores (BF16 operands, FP32 accumulation in tensor memory).
// The reference has no learned component; this is project design (see the header's
// cs_mlp_* functions for the network definition).
#include <cuda_bf16.h>

#include "../../include/clothstep.h"
#include "cs_internal.h"
#include "mlp.h"
#include "tc.cuh"

// ---------------------------------------------------------------------------------------
// Tile GEMM check: D[128 x N] = A[128 x K] B[N x K]^T through the same tcgen05 path the MLP
// layers use.  K in {16, 32, ..., 128}, N in {16, 32, ..., 128}.
__global__ void __launch_bounds__(128) cs_tc_gemm_check_kernel(const __nv_bfloat16* __restrict__ A,
                                                             const __nv_bfloat16* __restrict__ Bm, float* __restrict__ D,
                                                             int K, int N, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;                       // 128 x K bf16
    unsigned char* sB = smem + 128 * 128 * 2;       // N x K bf16
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * 128 * 128 * 2);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5;
    for (int k = 0; k < K; k++) tc::st_bf16(sA, 128, t, k, __bfloat162float(A[t * K + k]));
    for (int r = t; r < N; r += 128)
        for (int k = 0; k < K; k++) tc::st_bf16(sB, N, r, k, __bfloat162float(Bm[r * K + k]));
    if (t == 0) tc::mbar_init(bar, 1);
    if (warp == 0) tc::tmem_alloc(slot, 128);
    tc::fence_async_shared();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    if (t == 0) {
        tc::gemm_tile(tmem, tc::smem_u32(sA), tc::smem_u32(sB), K, N, false);
        tc::mma_commit(bar);
    }
    bool ok = tc::mbar_wait(bar, 0);
    tc::fence_after_sync();
    if (ok) {
        for (int c = 0; c < N / 16; c++) {
            float v[16];
            tc::tmem_ld16(tc::tmem_addr(tmem, warp, 16 * c), v);
            for (int i = 0; i < 16; i++) D[t * N + 16 * c + i] = v[i];
        }
    } else if (t == 0) {
        atomicExch(err, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

extern "C" cs_status cs_tc_gemm_check(const uint16_t* A, const uint16_t* B, float* D, int K, int N) {
    if (!A || !B || !D || K < 16 || K > 128 || K % 16 || N < 16 || N > 128 || N % 16) return CS_ERR_INVALID_ARG;
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float* dD = nullptr;
    int* derr = nullptr;
    cudaError_t e = cudaMalloc(&dA, 128 * K * 2);
    if (e == cudaSuccess) e = cudaMalloc(&dB, N * K * 2);
    if (e == cudaSuccess) e = cudaMalloc(&dD, 128 * N * 4);
    if (e == cudaSuccess) e = cudaMalloc(&derr, 4);
    if (e == cudaSuccess) e = cudaMemcpy(dA, A, 128 * K * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dB, B, N * K * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(derr, 0, 4);
    const int smem = 2 * 128 * 128 * 2 + 64;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(cs_tc_gemm_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) {
        cs_tc_gemm_check_kernel<<<1, 128, smem>>>(dA, dB, dD, K, N, derr);
        e = cudaDeviceSynchronize();
    }
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(D, dD, 128 * N * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, 4, cudaMemcpyDeviceToHost);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(derr);
    if (e != cudaSuccess) return CS_ERR_CUDA;
    return herr ? CS_ERR_TIMEOUT : CS_OK;
}

// ---------------------------------------------------------------------------------------
// Network (project design; the reference has no learned component).
//
// Per node i, 16 raw features (scale-free where the physics allows):
//   b_i / d_i (3), upper triangle of the diagonal block A_ii / d_i (6), v_i (3),
//   previous dv_i (3), m_i / d_i (1),   with d_i = trace(A_ii) / 3,
// standardised with the training set's mean and spread.  Two rounds of one-ring mean
// aggregation (agg(h)_i = mean of h_j over mesh neighbours j of i):
//   u1 = [x_i, agg(x)_i]              (32)  -> z1 = W1 u1 + b1 (64),  h1 = SiLU(z1)
//   u2 = [h1_i, agg(h1)_i]            (128) -> z2 = W2 u2 + b2 (64),  h2 = SiLU(z2)
//   z3 = W3 h2 + b3 (64), h3 = SiLU(z3);   y = W4 h3 + b4 (3)
//   prediction dv_i = previous dv_i + sigma_y * y + mu_y.
// MMA operands (u1, u2, h2 and the weights) are BF16; accumulation is FP32 in tensor memory;
// h1 is stored in BF16.  The three 64-wide layers and the backward products dz3 W3, dz2 W2
// run on tcgen05 with 128-node tiles; the 3-wide output layer runs on CUDA cores.
namespace {

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

struct Nbr {
    int beg, end, off;
};
__device__ __forceinline__ Nbr neighbours(const Batch& B, int node) {
    const SheetDesc& sh = B.sheets[B.node_sheet[node]];
    const int local = node - sh.node_off;
    Nbr r;
    r.beg = sh.nbr_off + B.nbr_ptr[sh.nbr_ptr_off + local];
    r.end = sh.nbr_off + B.nbr_ptr[sh.nbr_ptr_off + local + 1];
    r.off = sh.node_off;
    return r;
}

// Loads a row-major [rows x cols] BF16 weight matrix (optionally transposed) into a K-major
// canonical tile with R = rows (or cols if transposed) rows.
__device__ void load_weight_tile(const __nv_bfloat16* __restrict__ W, int rows, int cols, bool transpose,
                                 unsigned char* tile) {
    const int R = transpose ? cols : rows, K = transpose ? rows : cols;
    for (int e = threadIdx.x; e < R * K; e += blockDim.x) {
        const int r = e / K, k = e % K;
        const __nv_bfloat16 w = transpose ? W[k * cols + r] : W[r * cols + k];
        *reinterpret_cast<__nv_bfloat16*>(tile + tc::kmajor_offset(R, r, k)) = w;
    }
}

__device__ __forceinline__ void sync_tmem() {
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

}  // namespace

// Raw features of every node from the assembled system (diagonal block from the SELL panel
// of slot 0), the velocities and the previous dv held in B.warm.
__global__ void cs_mlp_features_kernel(Batch B, MlpDev M, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.N) return;
    const SheetDesc& sh = B.sheets[B.node_sheet[i]];
    const int local = i - sh.node_off;
    const int ts = B.row2slot[sh.row2slot_off + local];
    const SliceDesc& sd = B.slices[sh.slice_off + ts / CS_SLICE];
    const int lane = ts % CS_SLICE;
    const float* panel = B.A + (size_t)sd.panel0 * CS_PANEL_FLOATS;
    const float4 a0 = reinterpret_cast<const float4*>(panel)[lane];
    const float4 a1 = reinterpret_cast<const float4*>(panel + 128)[lane];
    const float a8 = panel[256 + lane];
    const float d = (a0.x + a1.x + a8) / 3.0f;
    const float id = d > 0.f ? 1.0f / d : 0.f;
    float* o = out + 16 * (size_t)i;
    o[0] = B.b[3 * i] * id;
    o[1] = B.b[3 * i + 1] * id;
    o[2] = B.b[3 * i + 2] * id;
    o[3] = a0.x * id;
    o[4] = a0.y * id;
    o[5] = a0.z * id;
    o[6] = a1.x * id;
    o[7] = a1.y * id;
    o[8] = a8 * id;
    o[9] = B.v[3 * i];
    o[10] = B.v[3 * i + 1];
    o[11] = B.v[3 * i + 2];
    o[12] = B.warm[3 * i];
    o[13] = B.warm[3 * i + 1];
    o[14] = B.warm[3 * i + 2];
    o[15] = B.mass[i] * id;
}

// Layer 1 over nodes [n0, n1): u1 = [x, agg(x)] -> h1 (BF16) and, when z1 != nullptr, z1.
__global__ void __launch_bounds__(128) cs_mlp_l1_kernel(Batch B, MlpDev M, const float* __restrict__ fsrc, int n0,
                                                      int n1, float* __restrict__ z1) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;              // 128 x 32 bf16: 8 KB
    unsigned char* sW = smem + 8192;       // 64 x 32 bf16: 4 KB
    float* sb = reinterpret_cast<float*>(smem + 12288);  // b1 (64), mu (16), sigma (16)
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 12288 + 512);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5;
    load_weight_tile(M.wb + MLP_W1, 64, 32, false, sW);
    for (int e = t; e < 64; e += 128) sb[e] = M.w[MLP_B1 + e];
    for (int e = t; e < 32; e += 128) sb[64 + e] = M.stats[e];
    if (t == 0) tc::mbar_init(bar, 1);
    if (warp == 0) tc::tmem_alloc(slot, 64);
    tc::fence_async_shared();
    sync_tmem();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    bool ok = true;
    const int ntiles = (n1 - n0 + 127) / 128;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int node = n0 + tile * 128 + t;
        const bool valid = node < n1;
        float u[32];
        if (valid) {
            // feature rows are 16 floats = 4 x 16 bytes
            const float4* x = reinterpret_cast<const float4*>(fsrc + 16 * (size_t)node);
            float acc[16];
#pragma unroll
            for (int g = 0; g < 4; g++) {
                const float4 xv = __ldg(x + g);
                u[4 * g] = (xv.x - sb[64 + 4 * g]) / sb[80 + 4 * g];
                u[4 * g + 1] = (xv.y - sb[65 + 4 * g]) / sb[81 + 4 * g];
                u[4 * g + 2] = (xv.z - sb[66 + 4 * g]) / sb[82 + 4 * g];
                u[4 * g + 3] = (xv.w - sb[67 + 4 * g]) / sb[83 + 4 * g];
            }
#pragma unroll
            for (int c = 0; c < 16; c++) acc[c] = 0.f;
            Nbr nb = neighbours(B, node);
            for (int k = nb.beg; k < nb.end; k++) {
                const float4* xj = reinterpret_cast<const float4*>(fsrc + 16 * (size_t)(B.nbr[k] + nb.off));
#pragma unroll
                for (int g = 0; g < 4; g++) {
                    const float4 xv = __ldg(xj + g);
                    acc[4 * g] += xv.x;
                    acc[4 * g + 1] += xv.y;
                    acc[4 * g + 2] += xv.z;
                    acc[4 * g + 3] += xv.w;
                }
            }
            const float inv = nb.end > nb.beg ? 1.0f / (nb.end - nb.beg) : 0.f;
#pragma unroll
            for (int c = 0; c < 16; c++) u[16 + c] = nb.end > nb.beg ? (acc[c] * inv - sb[64 + c]) / sb[80 + c] : 0.f;
        } else {
#pragma unroll
            for (int c = 0; c < 32; c++) u[c] = 0.f;
        }
#pragma unroll
        for (int g = 0; g < 4; g++) {
            __align__(16) __nv_bfloat16 ub[8];
#pragma unroll
            for (int c = 0; c < 8; c++) ub[c] = __float2bfloat16_rn(u[8 * g + c]);
            *reinterpret_cast<uint4*>(sA + tc::kmajor_offset(128, t, 8 * g)) = *reinterpret_cast<const uint4*>(ub);
        }
        tc::fence_async_shared();
        sync_tmem();
        if (t == 0) {
            tc::gemm_tile(tmem, tc::smem_u32(sA), tc::smem_u32(sW), 32, 64, false);
            tc::mma_commit(bar);
        }
        ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        tc::fence_after_sync();
        if (ok) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float zz[16];
                tc::tmem_ld16(tc::tmem_addr(tmem, warp, 16 * q), zz);
                if (valid) {
                    __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
                    for (int c = 0; c < 16; c++) {
                        const float z = zz[c] + sb[16 * q + c];
                        hb[c] = __float2bfloat16_rn(silu(z));
                        if (z1) z1[64 * (size_t)node + 16 * q + c] = z;
                    }
                    uint4* dst = reinterpret_cast<uint4*>(M.h1 + 64 * (size_t)node + 16 * q);
                    dst[0] = reinterpret_cast<uint4*>(hb)[0];
                    dst[1] = reinterpret_cast<uint4*>(hb)[1];
                }
            }
        } else if (t == 0) {
            atomicExch(M.err, 1);
        }
        sync_tmem();
    }
    if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

// Layers 2, 3 and the output over nodes [n0, n1).  Inference (z2 == nullptr): the prediction
// previous dv + sigma_y y + mu_y is written to pred (may alias B.warm).  Training: z2, z3, y.
__global__ void __launch_bounds__(128, 4) cs_mlp_l23_kernel(Batch B, MlpDev M, int n0, int n1, float* __restrict__ z2,
                                                       float* __restrict__ z3, float* __restrict__ yout,
                                                       float* pred) {
    // 51 KB, so that four CTAs (4 x 128 TMEM columns) share an SM: the u2 tile is free once
    // layer 2's MMA is done, and then holds h2 and layer 3's weights
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;                  // 128 x 128 bf16: 32 KB
    unsigned char* sH = smem;                  // after layer 2's MMA: 128 x 64, 16 KB
    unsigned char* sW3 = smem + 16384;         // after layer 2's MMA: 64 x 64, 8 KB
    unsigned char* sW2 = smem + 32768;         // 64 x 128: 16 KB
    float* sf = reinterpret_cast<float*>(smem + 49152);  // W4 (192), b2 (64), b3 (64), b4 (3), mu_y, sigma_y
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 49152 + 2048);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5;
    load_weight_tile(M.wb + MLP_W2, 64, 128, false, sW2);
    for (int e = t; e < 192; e += 128) sf[e] = __bfloat162float(M.wb[MLP_W4 + e]);
    for (int e = t; e < 64; e += 128) {
        sf[192 + e] = M.w[MLP_B2 + e];
        sf[256 + e] = M.w[MLP_B3 + e];
    }
    if (t < 3) {
        sf[320 + t] = M.w[MLP_B4 + t];
        sf[323 + t] = M.stats[32 + t];
        sf[326 + t] = M.stats[35 + t];
    }
    if (t == 0) tc::mbar_init(bar, 1);
    if (warp == 0) tc::tmem_alloc(slot, 128);
    tc::fence_async_shared();
    sync_tmem();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    bool ok = true;
    const int ntiles = (n1 - n0 + 127) / 128;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int node = n0 + tile * 128 + t;
        const bool valid = node < n1;
        // u2 = [h1_i, bf16(mean h1_j)]
        if (valid) {
            // rows of h1 are 64 BF16 = 8 x 16 bytes; a K-major tile keeps 8 consecutive k of a
            // row contiguous, so both the gathers and the tile stores move 16 bytes at a time
            const uint4* hi = reinterpret_cast<const uint4*>(M.h1 + 64 * (size_t)node);
            Nbr nb = neighbours(B, node);
            const float inv = nb.end > nb.beg ? 1.0f / (nb.end - nb.beg) : 0.f;
            // the first kNbr neighbours' rows, looked up once for the four quarters of the row;
            // their loads are issued kBatch at a time before the (ordered) additions
            constexpr int kNbr = 8, kBatch = 4;
            const int cnt = nb.end - nb.beg;
            const uint4* nrow[kNbr];
#pragma unroll
            for (int j = 0; j < kNbr; j++)
                nrow[j] = reinterpret_cast<const uint4*>(M.h1 + 64 * (size_t)(j < cnt ? B.nbr[nb.beg + j] + nb.off : node));
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float acc[16];
#pragma unroll
                for (int c = 0; c < 16; c++) acc[c] = 0.f;
                auto add_row = [&](const uint4& v0, const uint4& v1) {
                    const __nv_bfloat16* e0 = reinterpret_cast<const __nv_bfloat16*>(&v0);
                    const __nv_bfloat16* e1 = reinterpret_cast<const __nv_bfloat16*>(&v1);
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        acc[c] += __bfloat162float(e0[c]);
                        acc[8 + c] += __bfloat162float(e1[c]);
                    }
                };
#pragma unroll
                for (int j0 = 0; j0 < kNbr; j0 += kBatch) {
                    uint4 v0[kBatch], v1[kBatch];
#pragma unroll
                    for (int j = 0; j < kBatch; j++)
                        if (j0 + j < cnt) {
                            v0[j] = __ldg(nrow[j0 + j] + 2 * q);
                            v1[j] = __ldg(nrow[j0 + j] + 2 * q + 1);
                        }
#pragma unroll
                    for (int j = 0; j < kBatch; j++)
                        if (j0 + j < cnt) add_row(v0[j], v1[j]);
                }
                for (int k = nb.beg + kNbr; k < nb.end; k++) {
                    const uint4* hj = reinterpret_cast<const uint4*>(M.h1 + 64 * (size_t)(B.nbr[k] + nb.off) + 16 * q);
                    add_row(__ldg(hj), __ldg(hj + 1));
                }
                *reinterpret_cast<uint4*>(sA + tc::kmajor_offset(128, t, 16 * q)) = __ldg(hi + 2 * q);
                *reinterpret_cast<uint4*>(sA + tc::kmajor_offset(128, t, 16 * q + 8)) = __ldg(hi + 2 * q + 1);
#pragma unroll
                for (int hh = 0; hh < 2; hh++) {
                    __align__(16) __nv_bfloat16 ab[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) ab[c] = __float2bfloat16_rn(acc[8 * hh + c] * inv);
                    *reinterpret_cast<uint4*>(sA + tc::kmajor_offset(128, t, 64 + 16 * q + 8 * hh)) =
                        *reinterpret_cast<const uint4*>(ab);
                }
            }
        } else {
            const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
            for (int c = 0; c < 128; c += 8) *reinterpret_cast<uint4*>(sA + tc::kmajor_offset(128, t, c)) = zero;
        }
        tc::fence_async_shared();
        sync_tmem();
        if (t == 0) {
            tc::gemm_tile(tmem, tc::smem_u32(sA), tc::smem_u32(sW2), 128, 64, false);
            tc::mma_commit(bar);
        }
        ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        tc::fence_after_sync();
        if (!ok) break;
        // the u2 tile is free: layer 3's weights (row-major 64 x 64, this thread's 16 pairs, all
        // loads issued before the stores) into its second quarter; h2 goes into its first half
        {
            const uint32_t* w3g = reinterpret_cast<const uint32_t*>(M.wb + MLP_W3);
            uint32_t w3r[16];
#pragma unroll
            for (int i = 0; i < 16; i++) w3r[i] = __ldg(w3g + t + 128 * i);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int e = 2 * (t + 128 * i), r = e >> 6, k = e & 63;
                *reinterpret_cast<uint32_t*>(sW3 + tc::kmajor_offset(64, r, k)) = w3r[i];
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float zz[16];
            tc::tmem_ld16(tc::tmem_addr(tmem, warp, 16 * q), zz);
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const float z = zz[c] + sf[192 + 16 * q + c];
                if (z2 && valid) z2[64 * (size_t)node + 16 * q + c] = z;
                tc::st_bf16(sH, 128, t, 16 * q + c, valid ? silu(z) : 0.f);
            }
        }
        tc::fence_async_shared();
        sync_tmem();
        if (t == 0) {
            tc::gemm_tile(tmem + 64, tc::smem_u32(sH), tc::smem_u32(sW3), 64, 64, false);
            tc::mma_commit(bar);
        }
        ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        tc::fence_after_sync();
        if (!ok) break;
        float y0 = sf[320], y1 = sf[321], y2 = sf[322];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float zz[16];
            tc::tmem_ld16(tc::tmem_addr(tmem, warp, 64 + 16 * q), zz);
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const int j = 16 * q + c;
                const float z = zz[c] + sf[256 + j];
                if (z3 && valid) z3[64 * (size_t)node + j] = z;
                const float h = silu(z);
                y0 += sf[j] * h;
                y1 += sf[64 + j] * h;
                y2 += sf[128 + j] * h;
            }
        }
        if (valid) {
            if (yout) {
                yout[3 * (size_t)node] = y0;
                yout[3 * (size_t)node + 1] = y1;
                yout[3 * (size_t)node + 2] = y2;
            }
            if (pred) {
                const float p0 = B.warm[3 * node] + sf[326] * y0 + sf[323];
                const float p1 = B.warm[3 * node + 1] + sf[327] * y1 + sf[324];
                const float p2 = B.warm[3 * node + 2] + sf[328] * y2 + sf[325];
                pred[3 * node] = p0;
                pred[3 * node + 1] = p1;
                pred[3 * node + 2] = p2;
            }
        }
        sync_tmem();
    }
    if (!ok && t == 0) atomicExch(M.err, 1);
    sync_tmem();
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

// Backward through the output layer, layer 3 and layer 2 over nodes [n0, n1) (one training
// minibatch of whole sheets, ntot nodes).  With a target: loss = sum_i ||y_i - t_i||^2 / ntot
// with t_i = (target_i - mu_y) / sigma_y.  Without (target == nullptr): the energy-norm loss,
// whose gradient with respect to the prediction, ga A p - gb b, the energy kernels left (A p in
// M.dy, ga and gb per sheet in M.sheet_scale; dL/dy = sigma_y dL/dp); its value comes from those
// kernels.  Writes du2 (N x 128) for
// layer 1's backward and this CTA's gradient partials of W2, b2, W3, b3, W4, b4 and of the loss.
__global__ void __launch_bounds__(128) cs_mlp_bwd23_kernel(Batch B, MlpDev M, int n0, int n1,
                                                         const float* __restrict__ target) {
    extern __shared__ __align__(1024) unsigned char smem[];
    float* sDZ = reinterpret_cast<float*>(smem);                 // 128 x 65 fp32 (dz3, then dz2)
    float* sX = reinterpret_cast<float*>(smem + 33280);          // 128 x 65 fp32 (h3, then h2)
    __nv_bfloat16* sU = reinterpret_cast<__nv_bfloat16*>(smem + 66560);  // 128 x 136 bf16 (u2)
    unsigned char* sA = smem + 101376;                           // 128 x 64 bf16 MMA operand
    unsigned char* sW3t = smem + 117760;                         // 64 x 64 bf16 (W3^T)
    unsigned char* sW2t = smem + 125952;                         // 128 x 64 bf16 (W2^T)
    float* sf = reinterpret_cast<float*>(smem + 142336);         // W4 (192), mu_y, sigma_y, dy (128 x 4)
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 142336 + 2880);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    float* sDY = sf + 200;
    const int t = threadIdx.x, warp = t >> 5;
    load_weight_tile(M.wb + MLP_W3, 64, 64, true, sW3t);
    load_weight_tile(M.wb + MLP_W2, 64, 128, true, sW2t);
    for (int e = t; e < 192; e += 128) sf[e] = __bfloat162float(M.wb[MLP_W4 + e]);
    if (t < 3) {
        sf[192 + t] = M.stats[32 + t];
        sf[195 + t] = M.stats[35 + t];
    }
    if (t == 0) tc::mbar_init(bar, 1);
    if (warp == 0) tc::tmem_alloc(slot, 256);
    tc::fence_async_shared();
    sync_tmem();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    bool ok = true;
    const float scale = 2.0f / (float)max(n1 - n0, 1);
    // owned accumulators: row r of W2/W3 (columns half h), column t of W4, biases
    const int r = t >> 1, hf = t & 1;
    float acc2[64], acc3[32];
#pragma unroll
    for (int c = 0; c < 64; c++) acc2[c] = 0.f;
#pragma unroll
    for (int c = 0; c < 32; c++) acc3[c] = 0.f;
    float acc4[3] = {0.f, 0.f, 0.f}, accb2 = 0.f, accb3 = 0.f, accb4 = 0.f, loss = 0.f;
    const int ntiles = (n1 - n0 + 127) / 128;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int node = n0 + tile * 128 + t;
        const bool valid = node < n1;
        // 1. dy, h3, dz3
        float dy[3] = {0.f, 0.f, 0.f};
        if (valid && target) {
            for (int i = 0; i < 3; i++) {
                const float tt = (target[3 * (size_t)node + i] - sf[192 + i]) / sf[195 + i];
                const float d = M.y[3 * (size_t)node + i] - tt;
                loss += d * d;
                dy[i] = scale * d;
            }
        } else if (valid) {
            const int sh = B.node_sheet[node];
            const float ga = M.sheet_scale[2 * sh], gb = M.sheet_scale[2 * sh + 1];
            for (int i = 0; i < 3; i++)
                dy[i] = (ga * M.dy[3 * (size_t)node + i] - gb * B.b[3 * (size_t)node + i]) * sf[195 + i];
        }
        for (int i = 0; i < 3; i++) sDY[4 * t + i] = dy[i];
        for (int j = 0; j < 64; j++) {
            const float z = valid ? M.z3[64 * (size_t)node + j] : 0.f;
            const float h = valid ? silu(z) : 0.f;
            const float dh = dy[0] * sf[j] + dy[1] * sf[64 + j] + dy[2] * sf[128 + j];
            const float dz = valid ? dh * silu_grad(z) : 0.f;
            sX[65 * t + j] = h;
            sDZ[65 * t + j] = dz;
            tc::st_bf16(sA, 128, t, j, dz);
        }
        tc::fence_async_shared();
        sync_tmem();
        // 2. dh2 = bf16(dz3) W3 on the tensor cores, meanwhile dW4, db4, db3
        if (t == 0) {
            tc::gemm_tile(tmem, tc::smem_u32(sA), tc::smem_u32(sW3t), 64, 64, false);
            tc::mma_commit(bar);
        }
        if (t < 64) {
            for (int n = 0; n < 128; n++) {
                const float h = sX[65 * n + t];
                acc4[0] += sDY[4 * n] * h;
                acc4[1] += sDY[4 * n + 1] * h;
                acc4[2] += sDY[4 * n + 2] * h;
            }
        } else if (t < 67) {
            for (int n = 0; n < 128; n++) accb4 += sDY[4 * n + (t - 64)];
        }
        if (hf == 0)
            for (int n = 0; n < 128; n++) accb3 += sDZ[65 * n + r];
        __syncthreads();
        // 3. h2 = bf16(SiLU(z2)) and dW3
        for (int j = 0; j < 64; j++) sX[65 * t + j] = valid ? bf(silu(M.z2[64 * (size_t)node + j])) : 0.f;
        __syncthreads();
        for (int n = 0; n < 128; n++) {
            const float d = sDZ[65 * n + r];
#pragma unroll
            for (int c = 0; c < 32; c++) acc3[c] += d * sX[65 * n + 32 * hf + c];
        }
        ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        tc::fence_after_sync();
        if (!ok) break;
        // 4. dz2 = dh2 * SiLU'(z2); u2 rebuilt
        float dz2[64];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float dh[16];
            tc::tmem_ld16(tc::tmem_addr(tmem, warp, 16 * q), dh);
#pragma unroll
            for (int c = 0; c < 16; c++)
                dz2[16 * q + c] = valid ? dh[c] * silu_grad(M.z2[64 * (size_t)node + 16 * q + c]) : 0.f;
        }
        if (valid) {
            const __nv_bfloat16* hi = M.h1 + 64 * (size_t)node;
            Nbr nb = neighbours(B, node);
            const float inv = nb.end > nb.beg ? 1.0f / (nb.end - nb.beg) : 0.f;
            for (int j = 0; j < 64; j++) sU[136 * t + j] = hi[j];
            for (int q = 0; q < 4; q++) {
                float acc[16];
#pragma unroll
                for (int c = 0; c < 16; c++) acc[c] = 0.f;
                for (int k = nb.beg; k < nb.end; k++) {
                    const __nv_bfloat16* hj = M.h1 + 64 * (size_t)(B.nbr[k] + nb.off) + 16 * q;
#pragma unroll
                    for (int c = 0; c < 16; c++) acc[c] += __bfloat162float(hj[c]);
                }
#pragma unroll
                for (int c = 0; c < 16; c++) sU[136 * t + 64 + 16 * q + c] = __float2bfloat16_rn(acc[c] * inv);
            }
        } else {
            for (int j = 0; j < 128; j++) sU[136 * t + j] = __float2bfloat16_rn(0.f);
        }
        sync_tmem();  // every thread is done reading dz3 (sDZ) for dW3
#pragma unroll
        for (int j = 0; j < 64; j++) {
            sDZ[65 * t + j] = dz2[j];
            tc::st_bf16(sA, 128, t, j, dz2[j]);
        }
        tc::fence_async_shared();
        sync_tmem();
        // 5. du2 = bf16(dz2) W2 on the tensor cores, meanwhile dW2 and db2
        if (t == 0) {
            tc::gemm_tile(tmem + 64, tc::smem_u32(sA), tc::smem_u32(sW2t), 64, 128, false);
            tc::mma_commit(bar);
        }
        for (int n = 0; n < 128; n++) {
            const float d = sDZ[65 * n + r];
#pragma unroll
            for (int c = 0; c < 64; c++) acc2[c] += d * __bfloat162float(sU[136 * n + 64 * hf + c]);
            if (hf == 0) accb2 += d;
        }
        ok = __syncthreads_and(tc::mbar_wait(bar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        tc::fence_after_sync();
        if (!ok) break;
        // 6. du2 out
#pragma unroll
        for (int q = 0; q < 8; q++) {
            float du[16];
            tc::tmem_ld16(tc::tmem_addr(tmem, warp, 64 + 16 * q), du);
            if (valid) {
                float4* dst = reinterpret_cast<float4*>(M.du2 + 128 * (size_t)node + 16 * q);
#pragma unroll
                for (int c = 0; c < 4; c++) dst[c] = make_float4(du[4 * c], du[4 * c + 1], du[4 * c + 2], du[4 * c + 3]);
            }
        }
        sync_tmem();
    }
    if (!ok && t == 0) atomicExch(M.err, 1);
    sync_tmem();
    if (warp == 0) tc::tmem_dealloc(tmem, 256);
    // this CTA's partials
    float* gp = M.gpart + (size_t)blockIdx.x * MLP_P;
#pragma unroll
    for (int c = 0; c < 64; c++) gp[MLP_W2 + 128 * r + 64 * hf + c] = acc2[c];
#pragma unroll
    for (int c = 0; c < 32; c++) gp[MLP_W3 + 64 * r + 32 * hf + c] = acc3[c];
    if (hf == 0) {
        gp[MLP_B2 + r] = accb2;
        gp[MLP_B3 + r] = accb3;
    }
    if (t < 64)
        for (int i = 0; i < 3; i++) gp[MLP_W4 + 64 * i + t] = acc4[i];
    else if (t < 67)
        gp[MLP_B4 + t - 64] = accb4;
    // loss partial (fixed-order block sum)
    __shared__ float sl[128];
    sl[t] = loss;
    __syncthreads();
    if (t == 0) {
        float s = 0.f;
        for (int i = 0; i < 128; i++) s += sl[i];
        M.loss_part[blockIdx.x] = s / (float)max(n1 - n0, 1);
    }
}

// Backward into layer 1 over nodes [n0, n1): dh1_i = du2_i[0:64] + sum over neighbours j of
// du2_j[64:128] / deg_j (the transpose of the mean aggregation), dz1 = dh1 * SiLU'(z1),
// and this CTA's partials of W1, b1.
__global__ void __launch_bounds__(128) cs_mlp_bwd1_kernel(Batch B, MlpDev M, const float* __restrict__ fsrc, int n0,
                                                        int n1) {
    extern __shared__ __align__(16) float dyn[];
    float* sDZ = dyn;                 // 128 x 65
    float* sU = dyn + 128 * 65;       // 128 x 33
    float* sst = sU + 128 * 33;       // 32
    const int t = threadIdx.x;
    if (t < 32) sst[t] = M.stats[t];
    __syncthreads();
    const int r = t >> 1, hf = t & 1;
    float acc1[16], accb1 = 0.f;
#pragma unroll
    for (int c = 0; c < 16; c++) acc1[c] = 0.f;
    const int ntiles = (n1 - n0 + 127) / 128;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int node = n0 + tile * 128 + t;
        const bool valid = node < n1;
        if (valid) {
            Nbr nb = neighbours(B, node);
            float dh[64];
            for (int j = 0; j < 64; j++) dh[j] = M.du2[128 * (size_t)node + j];
            for (int k = nb.beg; k < nb.end; k++) {
                const int g = B.nbr[k] + nb.off;
                const SheetDesc& sh = B.sheets[B.node_sheet[g]];
                const int lg = g - sh.node_off;
                const int deg = B.nbr_ptr[sh.nbr_ptr_off + lg + 1] - B.nbr_ptr[sh.nbr_ptr_off + lg];
                const float w = 1.0f / (float)deg;
                for (int j = 0; j < 64; j++) dh[j] += M.du2[128 * (size_t)g + 64 + j] * w;
            }
            for (int j = 0; j < 64; j++) sDZ[65 * t + j] = dh[j] * silu_grad(M.z1[64 * (size_t)node + j]);
            // u1 = bf16([x, agg(x)]) as in the forward pass
            const float* x = fsrc + 16 * (size_t)node;
            float acc[16];
            for (int c = 0; c < 16; c++) {
                sU[33 * t + c] = bf((x[c] - sst[c]) / sst[16 + c]);
                acc[c] = 0.f;
            }
            for (int k = nb.beg; k < nb.end; k++) {
                const float* xj = fsrc + 16 * (size_t)(B.nbr[k] + nb.off);
                for (int c = 0; c < 16; c++) acc[c] += xj[c];
            }
            const float inv = nb.end > nb.beg ? 1.0f / (nb.end - nb.beg) : 0.f;
            for (int c = 0; c < 16; c++)
                sU[33 * t + 16 + c] = nb.end > nb.beg ? bf((acc[c] * inv - sst[c]) / sst[16 + c]) : 0.f;
        } else {
            for (int j = 0; j < 64; j++) sDZ[65 * t + j] = 0.f;
            for (int c = 0; c < 32; c++) sU[33 * t + c] = 0.f;
        }
        __syncthreads();
        for (int n = 0; n < 128; n++) {
            const float d = sDZ[65 * n + r];
#pragma unroll
            for (int c = 0; c < 16; c++) acc1[c] += d * sU[33 * n + 16 * hf + c];
            if (hf == 0) accb1 += d;
        }
        __syncthreads();
    }
    float* gp = M.gpart + (size_t)blockIdx.x * MLP_P;
#pragma unroll
    for (int c = 0; c < 16; c++) gp[MLP_W1 + 32 * r + 16 * hf + c] = acc1[c];
    if (hf == 0) gp[MLP_B1 + r] = accb1;
}

// Sums the per-CTA gradient partials in CTA order (deterministic), then one Adam step
// (Kingma & Ba 2015) on the FP32 master weights and a refresh of their BF16 copies.  With
// lr == 0 only the summed gradient is written to grad_out (gradient checks).
__global__ void cs_mlp_adam_kernel(MlpDev M, int ncta, float lr, float b1, float b2, float eps, int step,
                                   float* grad_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_P) return;
    float g = 0.f;
    for (int c = 0; c < ncta; c++) g += M.gpart[(size_t)c * MLP_P + p];
    if (grad_out) grad_out[p] = g;
    if (lr == 0.f) return;
    const float m = b1 * M.m[p] + (1.f - b1) * g;
    const float v = b2 * M.v[p] + (1.f - b2) * g * g;
    M.m[p] = m;
    M.v[p] = v;
    const float mh = m / (1.f - powf(b1, (float)step));
    const float vh = v / (1.f - powf(b2, (float)step));
    const float w = M.w[p] - lr * mh / (sqrtf(vh) + eps);
    M.w[p] = w;
    M.wb[p] = __float2bfloat16_rn(w);
}

// The same Adam update from a gradient held in a device buffer (summed or averaged over
// ranks by the caller).
__global__ void cs_mlp_adam_ext_kernel(MlpDev M, const float* __restrict__ grad, float lr, float b1, float b2,
                                       float eps, int step) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= MLP_P) return;
    const float g = grad[p];
    const float m = b1 * M.m[p] + (1.f - b1) * g;
    const float v = b2 * M.v[p] + (1.f - b2) * g * g;
    M.m[p] = m;
    M.v[p] = v;
    const float mh = m / (1.f - powf(b1, (float)step));
    const float vh = v / (1.f - powf(b2, (float)step));
    const float w = M.w[p] - lr * mh / (sqrtf(vh) + eps);
    M.w[p] = w;
    M.wb[p] = __float2bfloat16_rn(w);
}

// Training pair bookkeeping: the dataset slot receives the raw features of the current
// assembled system (with the previous dv held in B.warm) and, after the solve, the target
// dv - previous dv.
__global__ void cs_mlp_target_kernel(Batch B, const float* __restrict__ feat, float* __restrict__ target) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * B.N) return;
    const int node = i / 3, c = i % 3;
    target[i] = B.dv[i] - feat[16 * (size_t)node + 12 + c];
}

// Sums and sums of squares of the 16 features and 3 targets over nodes (FP64 per block).
__global__ void cs_mlp_moments_kernel(const float* __restrict__ feat, const float* __restrict__ target, long long n,
                                      double* __restrict__ out) {
    __shared__ double sh[38 * 128];
    double acc[38];
    for (int c = 0; c < 38; c++) acc[c] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        for (int c = 0; c < 16; c++) {
            double x = feat[16 * i + c];
            acc[c] += x;
            acc[19 + c] += x * x;
        }
        for (int c = 0; c < 3; c++) {
            double x = target[3 * i + c];
            acc[16 + c] += x;
            acc[35 + c] += x * x;
        }
    }
    for (int c = 0; c < 38; c++) sh[38 * threadIdx.x + c] = acc[c];
    __syncthreads();
    if (threadIdx.x < 38) {
        double s = 0.0;
        for (int k = 0; k < (int)blockDim.x; k++) s += sh[38 * k + threadIdx.x];
        out[38 * blockIdx.x + threadIdx.x] = s;
    }
}

// Adds this minibatch's loss (sum of the per-CTA partials, in CTA order) to *acc.
__global__ void cs_mlp_loss_acc_kernel(MlpDev M, int ncta, float* acc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float s = 0.f;
    for (int c = 0; c < ncta; c++) s += M.loss_part[c];
    *acc += s;
}

// ---------------------------------------------------------------------------------------
// Energy-norm training.  For a sheet with system A dv = b and solution dv*, the warm start the
// solver takes from a prediction p is its Galerkin multiple alpha p, alpha = p^T b / p^T A p
// (warm_scale), whose error in the energy norm is that of the zero guess times sin(theta),
// theta the angle between p and dv* in the A inner product.  The loss is therefore
//     L = sin^2(theta) = 1 - (p^T b)^2 / ((p^T A p)(dv*^T b))      (A dv* = b, in [0, 1]),
// scale-free and bounded; with u = p^T b, w = p^T A p, c = dv*^T b:
//     dL/dp = (2 u / (w c)) (alpha A p - b): one SpMV of the prediction.
// A minibatch's loss is the mean over its sheets.

namespace {
__device__ __forceinline__ double rwsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
}  // namespace

// Per row q = A p into M.dy over slices [sl0, sl1) (a warp per slice, its rows as the SELL
// panels hold them), and per slice the FP64 partials of p.b and p.A p.
__global__ void __launch_bounds__(128) cs_mlp_energy_kernel(Batch B, MlpDev M, int sl0, int sl1) {
    const int slice = sl0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (slice >= sl1) return;
    const SliceDesc sd = B.slices[slice];
    const int node_off = B.sheets[sd.sheet].node_off;
    const float* __restrict__ x = M.pred;
    double pb = 0.0, pq = 0.0;
    if (lane < sd.rows) {
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
        const float y[3] = {y0, y1, y2};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            M.dy[3 * row + c] = y[c];
            pb += (double)x[3 * row + c] * (double)B.b[3 * row + c];
            pq += (double)x[3 * row + c] * (double)y[c];
        }
    }
    pb = rwsum(pb);
    pq = rwsum(pq);
    if (lane == 0) {
        M.epart[2 * slice] = pb;
        M.epart[2 * slice + 1] = pq;
    }
}

// Per slice the FP64 partial of dv64 . b (the solution's energy dv*^T A dv* = dv*^T b).
__global__ void __launch_bounds__(128) cs_mlp_energy_norm_kernel(Batch B, MlpDev M, int sl0, int sl1) {
    const int slice = sl0 + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (slice >= sl1) return;
    const SliceDesc sd = B.slices[slice];
    double e = 0.0;
    if (lane < sd.rows) {
        const int row = sd.row0 + B.rowmap[sd.topo_slice * CS_SLICE + lane];
#pragma unroll
        for (int c = 0; c < 3; c++) e += B.dv64[3 * row + c] * (double)B.b[3 * row + c];
    }
    e = rwsum(e);
    if (lane == 0) {
        M.epart[2 * slice] = e;
        M.epart[2 * slice + 1] = 0.0;
    }
}

// A block per sheet of [s0, s1) sums its slices' partials in a fixed order.  mode 0: the
// solution's energy c into M.sheet_c; mode 1: with u = p.b, w = p.A p, the sheet's loss
// 1 - u^2 / (w c) and the two coefficients of its gradient dL/dp = ga A p - gb b,
// gb = 2 u / (w c (s1 - s0)), ga = gb u / w (a sheet with w <= 0 or c <= 0: loss 1, no gradient).
__global__ void __launch_bounds__(128) cs_mlp_energy_sheet_kernel(Batch B, MlpDev M, int s0, int s1, int mode) {
    __shared__ double sh[8];
    const int s = s0 + blockIdx.x;
    if (s >= s1) return;
    const SheetDesc& d = B.sheets[s];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < d.n_slices; i += blockDim.x) {
        a += M.epart[2 * (d.slice_off + i)];
        b += M.epart[2 * (d.slice_off + i) + 1];
    }
    a = rwsum(a);
    b = rwsum(b);
    if ((threadIdx.x & 31) == 0) {
        sh[2 * (threadIdx.x >> 5)] = a;
        sh[2 * (threadIdx.x >> 5) + 1] = b;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double u = (sh[0] + sh[2]) + (sh[4] + sh[6]);
    const double w = (sh[1] + sh[3]) + (sh[5] + sh[7]);
    if (mode == 0) {
        M.sheet_c[s] = u;
        return;
    }
    const double c = M.sheet_c[s];
    if (w > 0.0 && c > 0.0) {
        const double gb = 2.0 * u / (w * c * (double)(s1 - s0));
        M.sheet_loss[s] = (float)(1.0 - u * u / (w * c));
        M.sheet_scale[2 * s] = (float)(gb * u / w);
        M.sheet_scale[2 * s + 1] = (float)gb;
    } else {
        M.sheet_loss[s] = 1.f;
        M.sheet_scale[2 * s] = 0.f;
        M.sheet_scale[2 * s + 1] = 0.f;
    }
}

// *acc += the mean of the sheets' losses over [s0, s1), summed in sheet order.
__global__ void cs_mlp_energy_loss_kernel(MlpDev M, int s0, int s1, float* acc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float t = 0.f;
    for (int s = s0; s < s1; s++) t += M.sheet_loss[s];
    *acc += t / (float)max(s1 - s0, 1);
}
