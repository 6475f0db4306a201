// Allocation-free solve of one block-sparse system, for callers that cannot allocate device
// memory.  It has no counterpart in the reference.
//
// Who needs it: code that runs where cudaMalloc is unavailable or forbidden -- a host that
// owns every byte of device memory through its own allocator (game engines, simulation
// frameworks with fixed arenas), real-time loops that must not allocate for latency
// reasons, or plugins that may not grow the process's device footprint after start-up.
// Such a caller passes its system and output buffers; the solver's scratch vectors live
// in one fixed, file-scope device array instead of memory allocated per call.
//
// Limits and behaviour:
//   * at most CS_NOALLOC_MAX_ROWS (16384) block rows; larger systems are rejected with
//     CS_ERR_INVALID_ARG before anything is launched;
//   * the scratch array (kNoallocBytes, 2 MiB) is a static __device__ variable, so every GPU
//     that loads this library holds it until the process exits;
//   * every call on a device shares that one array and leaves its contents behind; the kernel
//     initialises everything it reads, so nothing has to start at zero between calls, but two
//     calls that overlap on the GPU (different streams, or concurrent host threads) race on
//     it and give wrong results -- serialise them;
//   * the array's device address is looked up with cudaGetSymbolAddress on the first call on
//     each device (with that device current) and cached; make that first call before any
//     stream capture begins;
//   * no cudaMalloc, cudaFree or allocating library routine is called.
//
// Algorithm: the same scheme as the batched solver (cs_step with CS_PREC_MIXED) for a single
// system: FP32 block-Jacobi PCG sweeps with FP64 dot products inside FP64 iterative refinement,
// run by one thread block so that every reduction is a deterministic block-level tree.
#include <mutex>

#include "../../include/clothstep.h"

namespace {

constexpr int kThreads = 1024;
// Per block row: dv64 (3 doubles), Pinv (9 floats), e, r, z, p, q (3 floats each).
constexpr size_t kRowBytes = 3 * sizeof(double) + 9 * sizeof(float) + 15 * sizeof(float);
constexpr size_t kNoallocBytes = 2u << 20;
static_assert((size_t)CS_NOALLOC_MAX_ROWS * kRowBytes + 256 <= kNoallocBytes, "scratch too small");

// The fixed scratch array.  Host code must not pass `g_scratch` itself to a kernel: on the host
// that name is only a stand-in, not a device address.  Its address comes from
// cudaGetSymbolAddress (scratch_address below).
static __device__ __align__(256) unsigned char g_scratch[kNoallocBytes];

struct Scratch {
    double* dv64;
    float *Pinv, *e, *r, *z, *p, *q;
    double* stats;  // [0] iterations, [1] relative residual, [2] status
};

__device__ Scratch carve(unsigned char* base, int n) {
    Scratch s;
    size_t off = 0;
    s.dv64 = reinterpret_cast<double*>(base + off);
    off += (size_t)3 * n * sizeof(double);
    s.Pinv = reinterpret_cast<float*>(base + off);
    off += (size_t)9 * n * sizeof(float);
    s.e = reinterpret_cast<float*>(base + off);
    off += (size_t)3 * n * sizeof(float);
    s.r = reinterpret_cast<float*>(base + off);
    off += (size_t)3 * n * sizeof(float);
    s.z = reinterpret_cast<float*>(base + off);
    off += (size_t)3 * n * sizeof(float);
    s.p = reinterpret_cast<float*>(base + off);
    off += (size_t)3 * n * sizeof(float);
    s.q = reinterpret_cast<float*>(base + off);
    s.stats = reinterpret_cast<double*>(base + kNoallocBytes - 256);
    return s;
}

// Deterministic block-wide sum of a double (fixed tree over kThreads threads).
__device__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        double t = l < (kThreads / 32) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (l == 0) sh[32] = t;
    }
    __syncthreads();
    return sh[32];
}

__global__ void __launch_bounds__(kThreads) noalloc_pcg_kernel(int n, int nnzb, const int32_t* __restrict__ rp,
                                                             const int32_t* __restrict__ ci,
                                                             const float* __restrict__ val,
                                                             const float* __restrict__ b, float* __restrict__ x,
                                                             double tol, int max_iters, unsigned char* base) {
    __shared__ double sh[33];
    __shared__ int bad;
    Scratch S = carve(base, n);
    const int t = threadIdx.x;
    if (t == 0) bad = 0;
    __syncthreads();
    // Row ranges and column indices are checked first; any entry outside [0, nnzb) x [0, n)
    // ends the call with CS_ERR_INVALID_ARG before the matrix or vectors are read.
    for (int i = t; i < n; i += kThreads) {
        int k0 = rp[i], k1 = rp[i + 1];
        if (k0 < 0 || k1 < k0 || k1 > nnzb) bad = 1;
        else
            for (int k = k0; k < k1; k++)
                if ((unsigned)ci[k] >= (unsigned)n) bad = 1;
    }
    __syncthreads();
    if (bad) {
        // x becomes NaN, so that a caller of the asynchronous form (which gets no status from
        // the device) cannot take stale contents of x for a solution
        for (int i = t; i < 3 * n; i += kThreads) x[i] = __int_as_float(0x7fc00000);
        if (t == 0) {
            S.stats[0] = 0;
            S.stats[1] = -1.0;
            S.stats[2] = CS_ERR_INVALID_ARG;
        }
        return;
    }
    // set-up: block-Jacobi inverses, dv64 = 0, ||b||
    double bb = 0.0;
    for (int i = t; i < n; i += kThreads) {
        double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (ci[k] == i)
                for (int c = 0; c < 9; c++) m[c] = val[9 * (size_t)k + c];
        double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
        double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
        double id = det != 0.0 ? 1.0 / det : 0.0;
        float* P = S.Pinv + 9 * (size_t)i;
        P[0] = (float)(c00 * id);
        P[1] = (float)((m[2] * m[7] - m[1] * m[8]) * id);
        P[2] = (float)((m[1] * m[5] - m[2] * m[4]) * id);
        P[3] = (float)(c01 * id);
        P[4] = (float)((m[0] * m[8] - m[2] * m[6]) * id);
        P[5] = (float)((m[2] * m[3] - m[0] * m[5]) * id);
        P[6] = (float)(c02 * id);
        P[7] = (float)((m[1] * m[6] - m[0] * m[7]) * id);
        P[8] = (float)((m[0] * m[4] - m[1] * m[3]) * id);
        for (int c = 0; c < 3; c++) {
            S.dv64[3 * i + c] = 0.0;
            S.e[3 * i + c] = 0.f;
            double bi = b[3 * i + c];
            bb += bi * bi;
        }
    }
    const double bn = sqrt(block_sum(bb, sh));
    const double inner_tol = 1e-4;
    int iters = 0;
    double rel = 0.0;
    int status = CS_ERR_NOT_CONVERGED;
    for (int sweep = 0; sweep < 64; sweep++) {
        // FP64 residual of dv64; start a sweep on it
        double rr = 0.0;
        __syncthreads();
        for (int i = t; i < n; i += kThreads) {
            double y[3] = {0, 0, 0};
            for (int k = rp[i]; k < rp[i + 1]; k++) {
                const float* A = val + 9 * (size_t)k;
                const int j = ci[k];
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) y[r] += (double)A[3 * r + c] * S.dv64[3 * j + c];
            }
            for (int r = 0; r < 3; r++) {
                double res = (double)b[3 * i + r] - y[r];
                S.r[3 * i + r] = (float)res;
                rr += res * res;
            }
        }
        const double res = sqrt(block_sum(rr, sh));
        rel = bn > 0.0 ? res / bn : 0.0;
        if (res <= tol * bn || bn == 0.0) {
            status = CS_OK;
            break;
        }
        if (iters >= max_iters) break;
        double rz = 0.0;
        for (int i = t; i < n; i += kThreads) {
            const float* P = S.Pinv + 9 * (size_t)i;
            float r0 = S.r[3 * i], r1 = S.r[3 * i + 1], r2 = S.r[3 * i + 2];
            float z0 = P[0] * r0 + P[1] * r1 + P[2] * r2;
            float z1 = P[3] * r0 + P[4] * r1 + P[5] * r2;
            float z2 = P[6] * r0 + P[7] * r1 + P[8] * r2;
            S.z[3 * i] = z0; S.z[3 * i + 1] = z1; S.z[3 * i + 2] = z2;
            S.p[3 * i] = z0; S.p[3 * i + 1] = z1; S.p[3 * i + 2] = z2;
            S.e[3 * i] = 0.f; S.e[3 * i + 1] = 0.f; S.e[3 * i + 2] = 0.f;
            rz += (double)r0 * z0 + (double)r1 * z1 + (double)r2 * z2;
        }
        rz = block_sum(rz, sh);
        while (iters < max_iters && rz > 0.0) {
            double pq = 0.0;
            for (int i = t; i < n; i += kThreads) {
                float y0 = 0.f, y1 = 0.f, y2 = 0.f;
                for (int k = rp[i]; k < rp[i + 1]; k++) {
                    const float* A = val + 9 * (size_t)k;
                    const int j = ci[k];
                    float p0 = S.p[3 * j], p1 = S.p[3 * j + 1], p2 = S.p[3 * j + 2];
                    y0 += A[0] * p0 + A[1] * p1 + A[2] * p2;
                    y1 += A[3] * p0 + A[4] * p1 + A[5] * p2;
                    y2 += A[6] * p0 + A[7] * p1 + A[8] * p2;
                }
                S.q[3 * i] = y0; S.q[3 * i + 1] = y1; S.q[3 * i + 2] = y2;
                pq += (double)S.p[3 * i] * y0 + (double)S.p[3 * i + 1] * y1 + (double)S.p[3 * i + 2] * y2;
            }
            pq = block_sum(pq, sh);
            if (!(pq > 0.0)) break;
            const float alpha = (float)(rz / pq);
            double rz2 = 0.0, rn = 0.0;
            for (int i = t; i < n; i += kThreads) {
                float r[3];
                for (int c = 0; c < 3; c++) {
                    S.e[3 * i + c] = __fmaf_rn(alpha, S.p[3 * i + c], S.e[3 * i + c]);
                    r[c] = __fmaf_rn(-alpha, S.q[3 * i + c], S.r[3 * i + c]);
                    S.r[3 * i + c] = r[c];
                }
                const float* P = S.Pinv + 9 * (size_t)i;
                float z0 = P[0] * r[0] + P[1] * r[1] + P[2] * r[2];
                float z1 = P[3] * r[0] + P[4] * r[1] + P[5] * r[2];
                float z2 = P[6] * r[0] + P[7] * r[1] + P[8] * r[2];
                S.z[3 * i] = z0; S.z[3 * i + 1] = z1; S.z[3 * i + 2] = z2;
                rz2 += (double)r[0] * z0 + (double)r[1] * z1 + (double)r[2] * z2;
                rn += (double)r[0] * r[0] + (double)r[1] * r[1] + (double)r[2] * r[2];
            }
            rz2 = block_sum(rz2, sh);
            rn = sqrt(block_sum(rn, sh));
            iters++;
            const float beta = (float)(rz2 / rz);
            rz = rz2;
            for (int i = t; i < n; i += kThreads)
                for (int c = 0; c < 3; c++) S.p[3 * i + c] = __fmaf_rn(beta, S.p[3 * i + c], S.z[3 * i + c]);
            __syncthreads();
            if (rn <= inner_tol * res || rn <= 0.5 * tol * bn) break;
        }
        for (int i = t; i < n; i += kThreads)
            for (int c = 0; c < 3; c++) S.dv64[3 * i + c] += (double)S.e[3 * i + c];
    }
    __syncthreads();
    for (int i = t; i < 3 * n; i += kThreads) x[i] = (float)S.dv64[i];
    if (t == 0) {
        S.stats[0] = iters;
        S.stats[1] = rel;
        S.stats[2] = status;
    }
}

std::mutex g_mutex;
unsigned char* g_addr[64] = {nullptr};

// Device address of g_scratch on the current device: looked up once per device with that
// device current, then cached.
cs_status scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= 64) return CS_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_addr[device]) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess || !ptr) return CS_ERR_CUDA;
        g_addr[device] = static_cast<unsigned char*>(ptr);
    }
    *out = g_addr[device];
    return CS_OK;
}

}  // namespace

extern "C" cs_status cs_solve_block_csr_noalloc(int n_rows, int nnzb, const int32_t* row_ptr, const int32_t* col,
                                               const float* val, const float* b, float* x, double tol,
                                               int max_iters, void* stream, int* iters, double* rel_residual) {
    if (n_rows <= 0 || n_rows > CS_NOALLOC_MAX_ROWS || nnzb <= 0) return CS_ERR_INVALID_ARG;
    if (!row_ptr || !col || !val || !b || !x || !(tol > 0.0) || max_iters < 0) return CS_ERR_INVALID_ARG;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return CS_ERR_NO_DEVICE;
    unsigned char* base = nullptr;
    cs_status st = scratch_address(device, &base);
    if (st != CS_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    noalloc_pcg_kernel<<<1, kThreads, 0, s>>>(n_rows, nnzb, row_ptr, col, val, b, x, tol, max_iters, base);
    if (cudaGetLastError() != cudaSuccess) return CS_ERR_CUDA;
    if (!iters && !rel_residual) return CS_OK;
    double stats[3];
    if (cudaMemcpyAsync(stats, base + kNoallocBytes - 256, sizeof(stats), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CS_ERR_CUDA;
    if (iters) *iters = (int)stats[0];
    if (rel_residual) *rel_residual = stats[1];
    return (cs_status)(int)stats[2];
}
