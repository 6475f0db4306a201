// Device-side lists for proximity terms (cs_set_proximities, cs_detect_proximities).
//
// Cloth::physicsStep receives every proximity of the scene and adds the terms of those
// holding its nodes, marking other nodes with index -1 (Cloth.cu:171-192).  Here a proximity
// becomes one instance per sheet holding one of its nodes (sheets in first-appearance order
// among its corners), and every row holding an instance's node gets the instance in an
// ascending per-row list, which cs_prox_row_kernel (forces.cu) walks each step in the
// reference's accumulation order.  Pairs of nodes outside the mesh pattern get a row-sorted
// side list of blocks (the reference's Eigen pattern grows instead).
//
// Kernels: count / expand (instances), row count / fill / sort (row lists), outside-pattern
// columns (count, then fill); a three-pass exclusive scan (block sums, one-block scan of the
// sums, per-block scan) turns counts into offsets.
#include "cs_internal.h"

// ---------------------------------------------------------------------------------------
// Exclusive scan of n ints in place; data[n] receives the total.

__global__ void __launch_bounds__(1024) cs_scan_sums_kernel(const int* data, int n, int* partial) {
    const long long base = (long long)blockIdx.x * CS_SCAN_ITEMS + 4LL * threadIdx.x;
    int s = 0;
    for (int j = 0; j < 4; j++)
        if (base + j < n) s += data[base + j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ int ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < 32; k++) t += ws[k];
        partial[blockIdx.x] = t;
    }
}

// one block: partial[] becomes exclusive block offsets; *total the sum
__global__ void __launch_bounds__(1024) cs_scan_partials_kernel(int* partial, int nb, int* total) {
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int b0 = 0; b0 < nb; b0 += 1024) {
        const int b = b0 + threadIdx.x;
        const int v = b < nb ? partial[b] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) ws[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int s = ws[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += u;
            }
            ws[lane] = s;
        }
        __syncthreads();
        if (b < nb) partial[b] = carry + (wid > 0 ? ws[wid - 1] : 0) + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += ws[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(1024) cs_scan_apply_kernel(int* data, int n, const int* partial) {
    const long long base = (long long)blockIdx.x * CS_SCAN_ITEMS + 4LL * threadIdx.x;
    int v[4], s = 0;
    for (int j = 0; j < 4; j++) {
        v[j] = base + j < n ? data[base + j] : 0;
        s += v[j];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    __shared__ int ws[32];
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int t = ws[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += u;
        }
        ws[lane] = t;
    }
    __syncthreads();
    int run = partial[blockIdx.x] + (wid > 0 ? ws[wid - 1] : 0) + incl - s;
    for (int j = 0; j < 4; j++) {
        if (base + j < n) data[base + j] = run;
        run += v[j];
    }
}

// ---------------------------------------------------------------------------------------

namespace {

// Distinct sheets among a proximity's batch nodes, in first-appearance order.
__device__ int prox_sheets(const Batch& B, const cs_proximity_desc& d, int sh[4]) {
    int k = 0;
    for (int i = 0; i < 4; i++) {
        if (d.nodes[i] < 0) continue;
        const int s = B.node_sheet[d.nodes[i]];
        bool seen = false;
        for (int j = 0; j < k; j++) seen |= sh[j] == s;
        if (!seen) sh[k++] = s;
    }
    return k;
}

// Is block (row, col) of one sheet on the mesh pattern?
__device__ bool on_pattern(const Batch& B, int row, int col) {
    const SheetDesc& sd = B.sheets[B.node_sheet[row]];
    const int* cp = B.tcsr_ptr + sd.csr_ptr_off;
    const int li = row - sd.node_off, lj = col - sd.node_off;
    int lo = cp[li], hi = cp[li + 1];
    const int end = hi;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (B.tcsr_col[mid] < lj) lo = mid + 1;
        else hi = mid;
    }
    return lo < end && B.tcsr_col[lo] == lj;
}

// Is corner a the first corner of the instance holding its (local) node?
__device__ __forceinline__ bool first_corner(const ProxInst& P, int a) {
    if (!((P.local >> a) & 1)) return false;
    for (int i = 0; i < a; i++)
        if (((P.local >> i) & 1) && P.node[i] == P.node[a]) return false;
    return true;
}

}  // namespace

__global__ void cs_prox_count_kernel(Batch B, const cs_proximity_desc* d, int n, int* icount) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int sh[4];
    icount[p] = prox_sheets(B, d[p], sh);
}

__global__ void cs_prox_expand_kernel(Batch B, const cs_proximity_desc* d, int n, const int* ioff, float thickness,
                                      ProxInst* inst, int* sheet_prox) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const cs_proximity_desc& D = d[p];
    int sh[4];
    const int k = prox_sheets(B, D, sh);
    for (int j = 0; j < k; j++) {
        ProxInst I;
        I.sheet = sh[j];
        I.local = 0;
        for (int i = 0; i < 4; i++) {
            I.node[i] = D.nodes[i];
            if (D.nodes[i] >= 0 && B.node_sheet[D.nodes[i]] == sh[j]) I.local |= 1 << i;
            for (int e = 0; e < 3; e++) {
                I.xe[i][e] = D.x[i][e];
                I.ve[i][e] = D.v[i][e];
            }
            I.me[i] = D.mass[i];
            I.w[i] = D.w[i];
        }
        I.free_mask = D.free_mask;
        I.thickness = thickness;
        for (int e = 0; e < 3; e++) I.n[e] = D.normal[e];
        I.mu = D.mu;
        I.stiffness = D.stiffness;
        inst[ioff[p] + j] = I;
        sheet_prox[sh[j]] = 1;
    }
}

__global__ void cs_prox_rowcount_kernel(const ProxInst* inst, int T, int* rowCount) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const ProxInst& P = inst[t];
    for (int a = 0; a < 4; a++)
        if (first_corner(P, a)) atomicAdd(&rowCount[P.node[a]], 1);
}

__global__ void cs_prox_rowfill_kernel(const ProxInst* inst, int T, const int* rowPtr, int* rowFill, int* rowInst) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const ProxInst& P = inst[t];
    for (int a = 0; a < 4; a++)
        if (first_corner(P, a)) {
            const int row = P.node[a];
            rowInst[rowPtr[row] + atomicAdd(&rowFill[row], 1)] = t;
        }
}

// Each row's instances ascending (insertion sort: the lists are short).
__global__ void cs_prox_rowsort_kernel(int N, const int* rowPtr, int* rowInst) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= N) return;
    const int q0 = rowPtr[row], q1 = rowPtr[row + 1];
    for (int q = q0 + 1; q < q1; q++) {
        const int v = rowInst[q];
        int r = q - 1;
        while (r >= q0 && rowInst[r] > v) {
            rowInst[r + 1] = rowInst[r];
            r--;
        }
        rowInst[r + 1] = v;
    }
}

// Columns of blocks outside the mesh pattern per row: with xptr null, their number into
// out[row]; otherwise the columns, ascending, into out[xptr[row]...].
__global__ void cs_prox_outside_kernel(Batch B, const int* rowPtr, const int* rowInst, const ProxInst* inst,
                                       const int* xptr, int* out) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= B.N) return;
    const int q0 = rowPtr[row], q1 = rowPtr[row + 1];
    // candidates: (q, b) in order; a column counts once, at its first candidate
    auto col_at = [&](int q, int b) -> int {
        const ProxInst& P = inst[rowInst[q]];
        if (!((P.local >> b) & 1)) return -1;
        return on_pattern(B, row, P.node[b]) ? -1 : P.node[b];
    };
    auto first = [&](int q, int b, int col) {
        for (int q2 = q0; q2 <= q; q2++)
            for (int b2 = 0; b2 < (q2 == q ? b : 4); b2++)
                if (col_at(q2, b2) == col) return false;
        return true;
    };
    int count = 0;
    for (int q = q0; q < q1; q++)
        for (int b = 0; b < 4; b++) {
            const int col = col_at(q, b);
            if (col < 0 || !first(q, b, col)) continue;
            if (xptr) out[xptr[row] + count] = col;
            count++;
        }
    if (!xptr) {
        out[row] = count;
        return;
    }
    int* seg = out + xptr[row];
    for (int i = 1; i < count; i++) {
        const int v = seg[i];
        int r = i - 1;
        while (r >= 0 && seg[r] > v) {
            seg[r + 1] = seg[r];
            r--;
        }
        seg[r + 1] = v;
    }
}
