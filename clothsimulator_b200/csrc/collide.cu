// The collision step on the device (cs_collision_step): Simulator::collisionStep as the
// reference's GPU path runs it after the implicit step (Simulator.cu:602-684).
//
// Each round: candidate face pairs from the contact grid over the start-of-step and current
// positions (contact.cu with ccd bounds, dilated by the collision thickness), then
//   cs_impact_kernel         per (pair, test) the shared-node and swept-box filters, the
//                            survivors compacted per block, then the continuous impact test
//                            of checkVertexFaceImpact / checkEdgeEdgeImpact
//                            (CollisionHelper.cu:61-136: the cubic for coplanarity along the
//                            linear trajectories, solveCubic / solveQuadratic /
//                            newtonsMethod :3-59, the distance and side at the root);
//   cs_impact_keys/gather_kernel  keys of the stable radix sorts by impact time (ties by node
//                            ids, type, index; the sorts are CUB's, in ctx.cu), then the gather;
//   cs_select_*_kernel       the independent impacts, earliest first, one per node
//                            (Simulator.cu:394-420), by rounds of per-node minima;
//   cs_opt_*_kernel          the impact zone's nodes (ascending), each impact's node slots,
//                            each node's constraint list in constraint order;
//   cs_opt_kernel            one CTA: CollisionOptimization (CollisionOptimization.cu) solved
//                            by Optimization::solve's augmented Lagrangian gradient descent
//                            (Optimization.cu:94-137).  Element terms are computed in
//                            parallel; every sum runs in the CPU loop's order on one thread,
//                            so the iterates are the FP32 CPU path's bit for bit.
// After the rounds, cs_collide_velocity_kernel sets v = (x - x0) / dt (Mesh.cu:238-247).
// Built without FMA contraction.
#include "cs_internal.h"

namespace {

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 ld(const float* p, int i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void st(float* p, int i, f3 a) {
    p[3 * i] = a.x;
    p[3 * i + 1] = a.y;
    p[3 * i + 2] = a.z;
}
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 scl(float s, f3 a) { return mk(s * a.x, s * a.y, s * a.z); }
// Vector.cuh:126-176 (dot and norm2 from zero, division by the reciprocal)
__device__ __forceinline__ float dot0(f3 a, f3 b) {
    float s = 0.0f;
    s += a.x * b.x;
    s += a.y * b.y;
    s += a.z * b.z;
    return s;
}
__device__ __forceinline__ f3 dvd(f3 a, float s) {
    const float inv = 1.0f / s;
    return mk(a.x * inv, a.y * inv, a.z * inv);
}
__device__ __forceinline__ f3 normalized(f3 a) { return dvd(a, sqrtf(dot0(a, a))); }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float mixed(f3 a, f3 b, f3 c) { return dot0(a, cross(b, c)); }  // MathHelper.cuh:43-45
__device__ __forceinline__ float mn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float ab(float x) { return x < 0.0f ? -x : x; }

// signedVertexFaceDistance / signedEdgeEdgeDistance (MathHelper.cu:38-69); false for INFINITY
__device__ bool signed_vf(f3 x, f3 y0, f3 y1, f3 y2, f3& n, float w[4], float& h) {
    n = cross(normalized(sub(y1, y0)), normalized(sub(y2, y0)));
    if (dot0(n, n) < 1e-6f) return false;
    n = normalized(n);
    h = dot0(sub(x, y0), n);
    const float b0 = mixed(sub(y1, x), sub(y2, x), n);
    const float b1 = mixed(sub(y2, x), sub(y0, x), n);
    const float b2 = mixed(sub(y0, x), sub(y1, x), n);
    w[0] = 1.0f;
    w[1] = -b0 / (b0 + b1 + b2);
    w[2] = -b1 / (b0 + b1 + b2);
    w[3] = -b2 / (b0 + b1 + b2);
    return true;
}
__device__ bool signed_ee(f3 x0, f3 x1, f3 y0, f3 y1, f3& n, float w[4], float& h) {
    n = cross(normalized(sub(x1, x0)), normalized(sub(y1, y0)));
    if (dot0(n, n) < 1e-6f) return false;
    n = normalized(n);
    h = dot0(sub(x0, y0), n);
    const float a0 = mixed(sub(y1, x1), sub(y0, x1), n);
    const float a1 = mixed(sub(y0, x0), sub(y1, x0), n);
    const float b0 = mixed(sub(x0, y1), sub(x1, y1), n);
    const float b1 = mixed(sub(x1, y0), sub(x0, y0), n);
    w[0] = a0 / (a0 + a1);
    w[1] = a1 / (a0 + a1);
    w[2] = -b0 / (b0 + b1);
    w[3] = -b1 / (b0 + b1);
    return true;
}

// CollisionHelper.cu:3-20
__device__ float newtons_method(float a, float b, float c, float d, float x0, int dir) {
    if (dir != 0) {
        const float y0 = d + x0 * (c + x0 * (b + x0 * a));
        const float ddy0 = 2.0f * b + x0 * (6.0f * a);
        x0 += (float)dir * sqrtf(ab(2.0f * y0 / ddy0));
    }
    for (int iter = 0; iter < 100; iter++) {
        const float y = d + x0 * (c + x0 * (b + x0 * a));
        const float dy = c + x0 * (2.0f * b + 3.0f * x0 * a);
        if (dy == 0) return x0;
        const float x1 = x0 - y / dy;
        if (ab(x0 - x1) < 1e-6f) return x0;
        x0 = x1;
    }
    return x0;
}

// CollisionHelper.cu:22-37
__device__ int solve_quadratic(float a, float b, float c, float x[2]) {
    const float d = b * b - 4.0f * a * c;
    if (d < 0.0f) {
        x[0] = -b / (2.0f * a);
        return 0;
    }
    const float q = -(b + (float)(b < 0.0f ? -1 : 1) * sqrtf(d)) * 0.5f;
    int i = 0;
    if (ab(a) > 1e-12f * ab(q)) x[i++] = q / a;
    if (ab(q) > 1e-12f * ab(c)) x[i++] = c / q;
    if (i == 2 && x[0] > x[1]) {
        const float t = x[0];
        x[0] = x[1];
        x[1] = t;
    }
    return i;
}

// CollisionHelper.cu:39-59.  Where solve_quadratic finds no root without writing one (both of
// its guards fail: a degenerate derivative), Newton's method starts from 0, as the oracle does
// (the reference reads an uninitialised value there).
__device__ int solve_cubic(float a, float b, float c, float d, float x[3]) {
    float xc[2] = {0.0f, 0.0f};
    const int n = solve_quadratic(3.0f * a, 2.0f * b, c, xc);
    if (n == 0) {
        x[0] = newtons_method(a, b, c, d, xc[0], 0);
        return 1;
    }
    if (n == 1) return solve_quadratic(b, c, d, x);
    const float yc[2] = {d + xc[0] * (c + xc[0] * (b + xc[0] * a)), d + xc[1] * (c + xc[1] * (b + xc[1] * a))};
    int i = 0;
    if (yc[0] * a >= 0.0f) x[i++] = newtons_method(a, b, c, d, xc[0], -1);
    if (yc[0] * yc[1] <= 0.0f) {
        const int closer = ab(yc[0]) < ab(yc[1]) ? 0 : 1;
        x[i++] = newtons_method(a, b, c, d, xc[closer], closer == 0 ? 1 : -1);
    }
    if (yc[1] * a <= 0.0f) x[i++] = newtons_method(a, b, c, d, xc[1], 1);
    return i;
}

// checkImpact (CollisionHelper.cu:61-110)
__device__ bool check_impact(int type, const f3 p[4], const f3 q[4], ImpactRec& r) {
    const f3 x0 = p[0];
    const f3 v0 = sub(q[0], x0);
    const f3 x1 = sub(p[1], x0), x2 = sub(p[2], x0), x3 = sub(p[3], x0);
    const f3 v1 = sub(sub(q[1], p[1]), v0), v2 = sub(sub(q[2], p[2]), v0), v3 = sub(sub(q[3], p[3]), v0);
    const float a0 = mixed(x1, x2, x3);
    const float a1 = mixed(v1, x2, x3) + mixed(x1, v2, x3) + mixed(x1, x2, v3);
    const float a2 = mixed(x1, v2, v3) + mixed(v1, x2, v3) + mixed(v1, v2, x3);
    const float a3 = mixed(v1, v2, v3);
    float t[3] = {0.0f, 0.0f, 0.0f};
    const int ns = solve_cubic(a3, a2, a1, a0, t);
    for (int i = 0; i < ns; i++) {
        if (t[i] < 0.0f || t[i] > 1.0f) continue;
        f3 y[4];
        for (int k = 0; k < 4; k++) y[k] = add(p[k], scl(t[i], sub(q[k], p[k])));  // Node::position
        f3 n;
        float w[4], h;
        bool inside;
        if (type == 0) {
            if (!signed_vf(y[0], y[1], y[2], y[3], n, w, h)) continue;
            inside = mn(-w[1], mn(-w[2], -w[3])) >= -1e-6f;
        } else {
            if (!signed_ee(y[0], y[1], y[2], y[3], n, w, h)) continue;
            inside = mn(mn(w[0], w[1]), mn(-w[2], -w[3])) >= -1e-6f;
        }
        if (dot0(n, add(add(scl(w[1], v1), scl(w[2], v2)), scl(w[3], v3))) > 0.0f) n = mk(-n.x, -n.y, -n.z);
        if (ab(h) < 1e-6f && inside) {
            r.type = type;
            r.t = t[i];
            for (int k = 0; k < 4; k++) r.w[k] = w[k];
            r.n[0] = n.x;
            r.n[1] = n.y;
            r.n[2] = n.z;
            return true;
        }
    }
    return false;
}

// Bounds of a node set over its start and current positions (Node/Face/Edge::bounds(ccd)).
__device__ void ccd_box(const Batch& B, const int* nodes, int k, float lo[3], float hi[3]) {
    for (int c = 0; c < 3; c++) {
        lo[c] = 3.0e38f;
        hi[c] = -3.0e38f;
    }
    for (int i = 0; i < k; i++) {
        const float* a = B.x + 3 * (size_t)nodes[i];
        const float* b = B.x0 + 3 * (size_t)nodes[i];
        for (int c = 0; c < 3; c++) {
            lo[c] = mn(mn(lo[c], a[c]), b[c]);
            hi[c] = mx(mx(hi[c], a[c]), b[c]);
        }
    }
}
// Bounds::overlap(b, thickness) (Bounds.cu:85-101): a against b dilated
__device__ bool overlap(const float alo[3], const float ahi[3], const float blo[3], const float bhi[3], float t) {
    for (int c = 0; c < 3; c++) {
        if (alo[c] > bhi[c] + t) return false;
        if (ahi[c] < blo[c] - t) return false;
    }
    return true;
}

// The swept-box filter of checkVertexFaceImpact / checkEdgeEdgeImpact (type 0: vertex-face,
// 1: edge-edge): false where the bounds of the two elements over the step stay apart.
__device__ bool impact_boxes_meet(const Batch& B, const Collide& K, int type, const int nodes[4]) {
    float alo[3], ahi[3], blo[3], bhi[3];
    if (type == 0) {
        ccd_box(B, nodes, 1, alo, ahi);
        ccd_box(B, nodes + 1, 3, blo, bhi);
    } else {
        ccd_box(B, nodes, 2, alo, ahi);
        ccd_box(B, nodes + 2, 2, blo, bhi);
    }
    return overlap(alo, ahi, blo, bhi, K.thickness);
}

// The continuous test of one element pair that passed the filters; an impact is appended.
__device__ void impact_test(const Batch& B, const Collide& K, int type, const int nodes[4]) {
    f3 p[4], q[4];
    for (int k = 0; k < 4; k++) {
        p[k] = ld(B.x0, nodes[k]);
        q[k] = ld(B.x, nodes[k]);
    }
    ImpactRec r;
    if (!check_impact(type, p, q, r)) return;
    for (int k = 0; k < 4; k++) r.nodes[k] = nodes[k];
    const int slot = atomicAdd(&K.counters[0], 1);
    if (slot < K.found_cap) K.found[slot] = r;
}

// The nodes of test k (0-5 vertex-face, 6-14 edge-edge) of candidate pair pr, or false where
// the two elements share a node (checkImpacts skips those, Simulator.cu:369-381).
__device__ bool impact_nodes(const Batch& B, const Contact& C, int2 pr, int k, int& type, int nodes[4]) {
    if (k < 6) {
        // vertex-face: corner k % 3 of one face against the other face
        const int f = k < 3 ? pr.x : pr.y, g = k < 3 ? pr.y : pr.x;
        const int4 y = B.face_nodes[f], z = B.face_nodes[g];
        const int i = k % 3;
        const int node = i == 0 ? y.x : i == 1 ? y.y : y.z;
        if (node == z.x || node == z.y || node == z.z) return false;
        type = 0;
        nodes[0] = node;
        nodes[1] = z.x;
        nodes[2] = z.y;
        nodes[3] = z.z;
        return true;
    }
    // edge-edge: edge i of the first face against edge j of the second
    const int4 fe = C.face_edges[pr.x], ge = C.face_edges[pr.y];
    const int i = (k - 6) / 3, j = (k - 6) % 3;
    const int4 a = C.edges[i == 0 ? fe.x : i == 1 ? fe.y : fe.z], b = C.edges[j == 0 ? ge.x : j == 1 ? ge.y : ge.z];
    if (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y) return false;
    type = 1;
    nodes[0] = a.x;
    nodes[1] = a.y;
    nodes[2] = b.x;
    nodes[3] = b.y;
    return true;
}

}  // namespace

// checkImpacts (Simulator.cu:369-381): per candidate pair its 6 vertex-face and 9 edge-edge
// tests.  Each block takes kImpactItems consecutive (pair, test) items: first every thread
// applies the cheap filters (shared nodes, swept boxes) to its items and queues the survivors
// in shared memory, then the block's threads share out the queued continuous tests, so the
// cubic solves run with full warps instead of beside threads that have nothing to do.  The
// impacts' order in `found` does not matter: the round sorts them by a total order.
constexpr int kImpactThreads = 256, kImpactPerThread = 8, kImpactItems = kImpactThreads * kImpactPerThread;
__global__ void __launch_bounds__(kImpactThreads) cs_impact_kernel(Batch B, Contact C, Collide K, int npairs) {
    __shared__ int4 qnodes[kImpactItems];
    __shared__ unsigned char qtype[kImpactItems];
    __shared__ int qcount;
    if (threadIdx.x == 0) qcount = 0;
    __syncthreads();
    const long long total = 15LL * npairs, base = (long long)blockIdx.x * kImpactItems;
    for (int j = 0; j < kImpactPerThread; j++) {
        const long long item = base + j * kImpactThreads + threadIdx.x;
        if (item >= total) break;
        const int2 pr = C.pairs[(int)(item / 15)];
        int type, nodes[4];
        if (!impact_nodes(B, C, pr, (int)(item % 15), type, nodes)) continue;
        if (!impact_boxes_meet(B, K, type, nodes)) continue;
        const int slot = atomicAdd(&qcount, 1);
        qnodes[slot] = make_int4(nodes[0], nodes[1], nodes[2], nodes[3]);
        qtype[slot] = (unsigned char)type;
    }
    __syncthreads();
    const int n = qcount;
    for (int q = threadIdx.x; q < n; q += kImpactThreads) {
        const int4 v = qnodes[q];
        const int nodes[4] = {v.x, v.y, v.z, v.w};
        impact_test(B, K, qtype[q], nodes);
    }
}

// Order of the found impacts: by time, then node ids, then type, then index (std::sort in
// Simulator::independentImpacts orders by time; the rest makes the order total).  A least-
// significant-first sequence of stable radix sorts (CUB, in ctx.cu) over the key parts: type,
// (n2, n3), n1, (t, n0).  t >= 0, so its IEEE bits order like its values once -0.0 (which the
// impact tests accept: it is not below 0, and the quadratic's c / q yields it for a start that
// is exactly coplanar) is taken as +0.0, as the oracle's comparison of times does; node ids
// are >= 0.  pass 0 also starts the permutation at the identity.
__global__ void cs_impact_keys_kernel(Collide K, int n, int pass, const int* __restrict__ perm,
                                      unsigned long long* __restrict__ key, int* __restrict__ perm_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int src = pass == 0 ? i : perm[i];
    if (pass == 0) perm_out[i] = i;
    const ImpactRec& r = K.found[src];
    unsigned long long k;
    if (pass == 0) k = (unsigned long long)(unsigned)r.type;
    else if (pass == 1) k = ((unsigned long long)(unsigned)r.nodes[2] << 32) | (unsigned)r.nodes[3];
    else if (pass == 2) k = (unsigned long long)(unsigned)r.nodes[1];
    else k = ((unsigned long long)(r.t == 0.0f ? 0u : __float_as_uint(r.t)) << 32) | (unsigned)r.nodes[0];
    key[i] = k;
}

__global__ void cs_impact_gather_kernel(Collide K, int n, const int* __restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) K.sorted[i] = K.found[perm[i]];
}

// independentImpacts (Simulator.cu:394-420) in parallel: the earliest-first greedy choice of
// impacts with disjoint nodes equals, round by round, the impacts that are the earliest live
// impact at each of their nodes; those are chosen, and the live impacts sharing a node with
// them drop out (the reference's GPU branch uses the same scheme, Simulator.cu:422-468).
__global__ void cs_select_init_kernel(Collide K, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i < n) K.alive[i] = 1;
    K.chosen[i] = 0;
}
__global__ void cs_select_reset_kernel(Collide K, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !K.alive[i]) return;
    for (int k = 0; k < 4; k++) K.nodemin[K.sorted[i].nodes[k]] = 0x7fffffff;
}
__global__ void cs_select_min_kernel(Collide K, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !K.alive[i]) return;
    for (int k = 0; k < 4; k++) atomicMin(&K.nodemin[K.sorted[i].nodes[k]], i);
}
__global__ void cs_select_choose_kernel(Collide K, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !K.alive[i]) return;
    const ImpactRec& r = K.sorted[i];
    bool first = true;
    for (int k = 0; k < 4; k++) first &= K.nodemin[r.nodes[k]] == i;
    if (!first) return;
    K.chosen[i] = 1;
    K.alive[i] = 0;
    for (int k = 0; k < 4; k++) K.used[r.nodes[k]] = 1;
}
__global__ void cs_select_drop_kernel(Collide K, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !K.alive[i]) return;
    const ImpactRec& r = K.sorted[i];
    bool hit = false;
    for (int k = 0; k < 4; k++) hit |= K.used[r.nodes[k]] != 0;
    if (hit) K.alive[i] = 0;
    else atomicAdd(&K.counters[1], 1);  // still live: another round
}
// The chosen impacts (exclusive offsets in chosen) appended in order; the node flags cleared.
__global__ void cs_select_write_kernel(Collide K, int n, int base, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const ImpactRec& r = K.sorted[i];
    if (K.chosen[i + 1] > K.chosen[i] && base + K.chosen[i] < cap) K.all[base + K.chosen[i]] = r;
    for (int k = 0; k < 4; k++) K.used[r.nodes[k]] = 0;
}

// The projection's nodes: marked, then (after an exclusive scan of mark) listed ascending.
__global__ void cs_opt_mark_kernel(Collide K, int nc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * nc) return;
    K.mark[K.all[t >> 2].nodes[t & 3]] = 1;
}
__global__ void cs_opt_nodes_kernel(Collide K, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (K.mark[i + 1] > K.mark[i]) K.nodes[K.mark[i]] = i;
}
__global__ void cs_opt_idx_kernel(Collide K, int nc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * nc) return;
    const int slot = K.mark[K.all[t >> 2].nodes[t & 3]];
    K.idx[t] = slot;
    atomicAdd(&K.nptr[slot], 1);
}
__global__ void cs_opt_fill_kernel(Collide K, int nc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * nc) return;
    const int slot = K.idx[t];
    K.nlist[K.nptr[slot] + atomicAdd(&K.nfill[slot], 1)] = t;
}
__global__ void cs_opt_sort_kernel(Collide K, int nn) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nn) return;
    const int q0 = K.nptr[s], q1 = K.nptr[s + 1];
    for (int q = q0 + 1; q < q1; q++) {
        const int v = K.nlist[q];
        int r = q - 1;
        while (r >= q0 && K.nlist[r] > v) {
            K.nlist[r + 1] = K.nlist[r];
            r--;
        }
        K.nlist[r + 1] = v;
    }
}

namespace {
constexpr float kMu = 1e3f;          // Optimization::solve (Optimization.cu:96)
constexpr float kEpsS = 1e-12f;      // Optimization.cuh:16
constexpr float kEpsF = 1e-10f;      // Optimization.cuh:17
constexpr int kMaxOptIterations = 100;

// CollisionOptimization::constraint (CollisionOptimization.cu:91-103)
__device__ float constraint(const Collide& K, const float* x, int c) {
    const ImpactRec& r = K.all[c];
    const f3 n = mk(r.n[0], r.n[1], r.n[2]);
    float a = -K.thickness;
    for (int k = 0; k < 4; k++) a += r.w[k] * dot0(n, ld(x, K.idx[4 * c + k]));
    return a;
}

// Optimization::value's terms at x: per node mass |x - x1|^2, per constraint its clamped
// violation (coef) and 0.5 mu coef^2.
__device__ void value_terms(const Batch& B, const Collide& K, const float* x, int nn, int nc) {
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
        const int node = K.nodes[i];
        const f3 d = sub(ld(x, i), ld(K.x1, node));
        K.nterm[i] = B.mass[node] * dot0(d, d);
    }
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        const float co = mn(constraint(K, x, c) + K.lambda[c] / kMu, 0.0f);  // clampViolation(x, +1)
        K.coef[c] = co;
        // skipped terms (coefficient 0) enter as +0: the running sum is >= +0, so adding +0
        // leaves it unchanged, bit for bit
        K.cterm[c] = co != 0.0f ? 0.5f * kMu * (co * co) : 0.0f;
    }
}

constexpr int kStage = 8192;  // floats staged in shared memory per chunk of a sequential sum

// acc + src[0] + src[1] + ... in that order (the CPU loop's), by thread 0, with the terms
// staged through shared memory by the whole block; every thread calls it; the result is
// thread 0's.
__device__ float ordered_sum(const float* src, int n, float acc, float* stage) {
    for (int base = 0; base < n; base += kStage) {
        const int m = min(kStage, n - base);
        for (int i = threadIdx.x; i < m; i += blockDim.x) stage[i] = src[base + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            int i = 0;
            for (; i + 8 <= m; i += 8) {
                float v[8];
#pragma unroll
                for (int k = 0; k < 8; k++) v[k] = stage[i + k];
#pragma unroll
                for (int k = 0; k < 8; k++) acc += v[k];
            }
            for (; i < m; i++) acc += stage[i];
        }
        __syncthreads();
    }
    return acc;
}

// Optimization::value (Optimization.cu:24-35) from those terms: the objective's sum, scaled,
// then the constraints' terms, in the CPU loop's order (thread 0's result).
__device__ float value_sum(const Collide& K, int nn, int nc, float invMass, float* stage) {
    float a = ordered_sum(K.nterm, nn, 0.0f, stage);
    a = 0.5f * a * invMass;  // meaningful in thread 0
    return ordered_sum(K.cterm, nc, a, stage);
}
}  // namespace

// One CTA: Optimization::solve (Optimization.cu:94-137) of CollisionOptimization over the
// accumulated impacts; the result is written back into B.x.
__global__ void __launch_bounds__(1024) cs_opt_kernel(Batch B, Collide K, int nn, int nc) {
    __shared__ float sf, sft, ss, sg2, sInv;
    __shared__ int sgo;
    __shared__ float stage[kStage];
    const int tid = threadIdx.x, T = blockDim.x;
    for (int i = tid; i < nn; i += T) st(K.cur, i, ld(B.x, K.nodes[i]));
    for (int c = tid; c < nc; c += T) K.lambda[c] = 0.0f;
    if (tid == 0) {
        // CollisionOptimization.cu:22-35: the mean inverse mass
        float inv = 0.0f;
        for (int i = 0; i < nn; i++) inv += 1.0f / B.mass[K.nodes[i]];
        sInv = inv / (float)nn;
        ss = 1e-3f * (float)nn;
    }
    __syncthreads();
    const float invMass = sInv;
    for (int iter = 0; iter < kMaxOptIterations; iter++) {
        // valueAndGradient (Optimization.cu:51-63) at cur
        value_terms(B, K, K.cur, nn, nc);
        __syncthreads();
        for (int i = tid; i < nn; i += T) {
            const int node = K.nodes[i];
            f3 g = scl(invMass * B.mass[node], sub(ld(K.cur, i), ld(K.x1, node)));
            for (int q = K.nptr[i]; q < K.nptr[i + 1]; q++) {
                const int c = K.nlist[q] >> 2, k = K.nlist[q] & 3;
                const float co = K.coef[c];
                if (co == 0.0f) continue;
                const ImpactRec& r = K.all[c];
                g = add(g, scl((kMu * co) * r.w[k], mk(r.n[0], r.n[1], r.n[2])));
            }
            st(K.grad, i, g);
            K.gterm[i] = dot0(g, g);
        }
        __syncthreads();
        {
            const float f = value_sum(K, nn, nc, invMass, stage);
            const float g2 = ordered_sum(K.gterm, nn, 0.0f, stage);
            if (tid == 0) {
                sf = f;
                sg2 = g2;
                ss /= 0.7f;
            }
        }
        __syncthreads();
        // backtracking line search
        for (;;) {
            if (tid == 0) ss *= 0.7f;
            __syncthreads();
            const float s = ss;
            for (int i = tid; i < nn; i += T) st(K.next, i, sub(ld(K.cur, i), scl(s, ld(K.grad, i))));
            __syncthreads();
            value_terms(B, K, K.next, nn, nc);
            __syncthreads();
            const float ft = value_sum(K, nn, nc, invMass, stage);
            if (tid == 0) {
                sft = ft;
                sgo = (ft >= sf - 0.5f * s * sg2 && s >= kEpsS && ab(sf - ft) >= kEpsF) ? 1 : 0;
            }
            __syncthreads();
            if (!sgo) break;
        }
        if (ss < kEpsS || ab(sf - sft) < kEpsF) break;
        for (int i = tid; i < nn; i += T) st(K.cur, i, ld(K.next, i));
        __syncthreads();
        // updateMultiplier (Optimization.cu:85-92)
        for (int c = tid; c < nc; c += T) K.lambda[c] = mn(K.lambda[c] + kMu * constraint(K, K.cur, c), 0.0f);
        __syncthreads();
    }
    __syncthreads();
    for (int i = tid; i < nn; i += T) st(B.x, K.nodes[i], ld(K.cur, i));
}

// Mesh::updateVelocities (Mesh.cu:238-247): v = (x - x0) * (1 / dt)
__global__ void cs_collide_velocity_kernel(Batch B, float invDt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * B.N) return;
    B.v[i] = (B.x[i] - B.x0[i]) * invDt;
}
