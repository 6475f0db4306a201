// Proximity detection on the device: the proximities Simulator::physicsStep finds before
// stepping the cloths (Simulator.cu:571-586 -> findProximitiesGpu, Simulator.cu:300-349).
//
// The reference builds a BVH per cloth, traverses face pairs whose bounds overlap after
// dilating one by 2 x repulsionThickness (BVH.cu, BVHHelper.cu, BVHNode.cu:40-63), tests
// every pair's vertex-face and edge-edge combinations (checkProximitiesGpu,
// PhysicsHelper.cu:20-113), then sorts and min-reduces the candidates per (node | edge |
// face, side) key with thrust and builds one Proximity per surviving key (:115-150,
// Proximity.cu:5-21).  Which face pairs are tested does not depend on the tree, only on the
// bounds, so this file finds them with a spatial hash grid instead (no sort, no tree build):
//
//   cs_contact_face_kernel   thread per face: normal (Face::update, Face.cu:124-132), bounds,
//                            largest extent (sets the cell size)
//   cs_contact_node_kernel   thread per node: normal (Mesh::updateNodeGeometries,
//                            Mesh.cu:182-203, faces in index order)
//   cs_contact_grid_kernel   thread per face: pushes the face onto the bucket of every cell
//                            its bounds touch (lock-free singly linked lists; buckets by the
//                            spatial hash of Teschner et al. 2003 with a final bit mix)
//   cs_contact_pair_kernel   thread per face f: walks the cells of its dilated bounds and
//                            appends each face g > f of its collision group whose bounds
//                            overlap, once per pair (in the lowest cell the two share)
//   cs_contact_vf/ee_kernel  thread per (pair, vertex-face test) and per (pair, edge-edge
//                            test): every lane of a warp runs the same test
//   cs_contact_count/scan/write_kernel: ordered compaction of the admitted keys (distance
//                            below 2 x repulsionThickness) into proximity records, in the
//                            reference's output order: node keys, edge keys, face keys
//
// The min-reduction is a 64-bit atomicMin on (distance bits << 32 | other element id): the
// distance is non-negative, so its IEEE bits order like the value, and ties break by the
// other element's id, whatever order the tests run in.  All arithmetic is FP32 in the
// reference's operation order; this file is built without FMA contraction.
#include "cs_internal.h"

namespace {

struct v3 {
    float x, y, z;
};
__device__ __forceinline__ v3 mk3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ v3 ldx(const float* p, int i) { return mk3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ v3 sub(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 add(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 scl(float s, v3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ v3 neg(v3 a) { return mk3(-a.x, -a.y, -a.z); }
// Vector.cuh:126-158: dot and norm2 accumulate from zero; division multiplies by the reciprocal
__device__ __forceinline__ float dot0(v3 a, v3 b) {
    float s = 0.0f;
    s += a.x * b.x;
    s += a.y * b.y;
    s += a.z * b.z;
    return s;
}
__device__ __forceinline__ v3 dvd(v3 a, float s) {
    const float inv = 1.0f / s;
    return mk3(a.x * inv, a.y * inv, a.z * inv);
}
__device__ __forceinline__ v3 normalized(v3 a) { return dvd(a, sqrtf(dot0(a, a))); }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// MathHelper.cuh:15-42
__device__ __forceinline__ float mn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float ab(float x) { return x < 0.0f ? -x : x; }
__device__ __forceinline__ v3 fnrm(const Contact& C, int f) { return ldx(C.fn, f); }
__device__ __forceinline__ v3 nnrm(const Contact& C, int i) { return ldx(C.nn, i); }

// signedVertexFaceDistance (MathHelper.cu:38-52); false where the reference returns INFINITY
__device__ bool signed_vf(v3 x, v3 y0, v3 y1, v3 y2, v3& n, float w[4], float& h) {
    n = cross(normalized(sub(y1, y0)), normalized(sub(y2, y0)));
    if (dot0(n, n) < 1e-6f) return false;
    n = normalized(n);
    h = dot0(sub(x, y0), n);
    const float b0 = dot0(sub(y1, x), cross(sub(y2, x), n));
    const float b1 = dot0(sub(y2, x), cross(sub(y0, x), n));
    const float b2 = dot0(sub(y0, x), cross(sub(y1, x), n));
    w[0] = 1.0f;
    w[1] = -b0 / (b0 + b1 + b2);
    w[2] = -b1 / (b0 + b1 + b2);
    w[3] = -b2 / (b0 + b1 + b2);
    return true;
}

// signedEdgeEdgeDistance (MathHelper.cu:54-69)
__device__ bool signed_ee(v3 x0, v3 x1, v3 y0, v3 y1, v3& n, float w[4], float& h) {
    n = cross(normalized(sub(x1, x0)), normalized(sub(y1, y0)));
    if (dot0(n, n) < 1e-6f) return false;
    n = normalized(n);
    h = dot0(sub(x0, y0), n);
    const float a0 = dot0(sub(y1, x1), cross(sub(y0, x1), n));
    const float a1 = dot0(sub(y0, x0), cross(sub(y1, x0), n));
    const float b0 = dot0(sub(x0, y1), cross(sub(x1, y1), n));
    const float b1 = dot0(sub(x1, y0), cross(sub(x0, y0), n));
    w[0] = a0 / (a0 + a1);
    w[1] = a1 / (a0 + a1);
    w[2] = -b0 / (b0 + b1);
    w[3] = -b1 / (b0 + b1);
    return true;
}

// inEdge (PhysicsHelper.cu:3-18): the point at w along edge e0 lies on the inner side of each
// face adjacent to edge e1.
__device__ bool in_edge(const Batch& B, const Contact& C, float w, int e0, int e1) {
    const int4 a = C.edges[e0], b = C.edges[e1];
    const v3 x = add(scl(1.0f - w, ldx(B.x, a.x)), scl(w, ldx(B.x, a.y)));
    bool in = true;
    for (int i = 0; i < 2; i++) {
        const int face = i == 0 ? b.z : b.w;
        if (face < 0) continue;
        const int node0 = i == 0 ? b.x : b.y, node1 = i == 0 ? b.y : b.x;
        const v3 e = sub(ldx(B.x, node1), ldx(B.x, node0));
        const v3 r = sub(x, ldx(B.x, node0));
        in &= (dot0(e, cross(fnrm(C, face), r)) >= 0.0f);
    }
    return in;
}

__device__ __forceinline__ unsigned long long pack(float d, int other) {
    if (d == 0.0f) d = 0.0f;  // -0 ties with +0, as the reference's comparison has it
    return ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)other;
}

// checkVertexFaceProximity (Simulator.cu:198-229, PhysicsHelper.cu:20-53)
__device__ void check_vf(const Batch& B, const Contact& C, int node, int face) {
    const int4 y = B.face_nodes[face];
    if (node == y.x || node == y.y || node == y.z) return;
    v3 n;
    float w[4], h;
    if (!signed_vf(ldx(B.x, node), ldx(B.x, y.x), ldx(B.x, y.y), ldx(B.x, y.z), n, w, h)) return;
    const float d = ab(h);
    if (!(mn(-w[1], mn(-w[2], -w[3])) >= 1e-6f)) return;
    const int sideN = dot0(n, nnrm(C, node)) >= 0.0f ? 0 : 1;
    atomicMin(&C.keys[2 * (size_t)node + sideN], pack(d, face));
    const int sideF = -dot0(n, fnrm(C, face)) >= 0.0f ? 0 : 1;
    atomicMin(&C.keys[2 * ((size_t)B.N + C.E + face) + sideF], pack(d, node));
}

// checkEdgeEdgeProximity (Simulator.cu:231-261, PhysicsHelper.cu:55-89)
__device__ void check_ee(const Batch& B, const Contact& C, int e0, int e1) {
    const int4 a = C.edges[e0], b = C.edges[e1];
    if (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y) return;
    v3 n;
    float w[4], h;
    if (!signed_ee(ldx(B.x, a.x), ldx(B.x, a.y), ldx(B.x, b.x), ldx(B.x, b.y), n, w, h)) return;
    const float d = ab(h);
    if (!(mn(mn(w[0], w[1]), mn(-w[2], -w[3])) >= 1e-6f && in_edge(B, C, w[1], e0, e1) && in_edge(B, C, -w[3], e1, e0)))
        return;
    const int side0 = dot0(n, add(nnrm(C, a.x), nnrm(C, a.y))) >= 0.0f ? 0 : 1;
    atomicMin(&C.keys[2 * ((size_t)B.N + e0) + side0], pack(d, e1));
    const int side1 = -dot0(n, add(nnrm(C, b.x), nnrm(C, b.y))) >= 0.0f ? 0 : 1;
    atomicMin(&C.keys[2 * ((size_t)B.N + e1) + side1], pack(d, e0));
}

__device__ __forceinline__ float cell_size(const Contact& C) {
    return (__uint_as_float(C.ext[0]) + 2.0f * C.dilate) * 1.0001f + 1e-30f;
}
__device__ __forceinline__ int cell_of(float v, float c) {
    return (int)fminf(fmaxf(floorf(v / c), -1073741824.0f), 1073741824.0f);
}
__device__ __forceinline__ unsigned bucket(const Contact& C, int group, int ix, int iy, int iz) {
    unsigned h = ((unsigned)ix * 73856093u) ^ ((unsigned)iy * 19349663u) ^ ((unsigned)iz * 83492791u) ^
                 ((unsigned)group * 2654435761u);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h & ((1u << C.hash_bits) - 1u);
}

}  // namespace

__global__ void __launch_bounds__(128) cs_contact_face_kernel(Batch B, Contact C) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= B.F) return;
    const int4 y = B.face_nodes[f];
    const v3 a = ldx(B.x, y.x), b = ldx(B.x, y.y), c = ldx(B.x, y.z);
    const v3 n = normalized(cross(sub(b, a), sub(c, a)));
    C.fn[3 * (size_t)f] = n.x;
    C.fn[3 * (size_t)f + 1] = n.y;
    C.fn[3 * (size_t)f + 2] = n.z;
    float lo[3] = {mn(mn(a.x, b.x), c.x), mn(mn(a.y, b.y), c.y), mn(mn(a.z, b.z), c.z)};
    float hi[3] = {mx(mx(a.x, b.x), c.x), mx(mx(a.y, b.y), c.y), mx(mx(a.z, b.z), c.z)};
    if (C.ccd) {  // Face::bounds(ccd) (Face.cu:94-103): the start-of-step positions too
        const v3 a0 = ldx(B.x0, y.x), b0 = ldx(B.x0, y.y), c0 = ldx(B.x0, y.z);
        const float l0[3] = {mn(mn(a0.x, b0.x), c0.x), mn(mn(a0.y, b0.y), c0.y), mn(mn(a0.z, b0.z), c0.z)};
        const float h0[3] = {mx(mx(a0.x, b0.x), c0.x), mx(mx(a0.y, b0.y), c0.y), mx(mx(a0.z, b0.z), c0.z)};
        for (int k = 0; k < 3; k++) {
            lo[k] = mn(lo[k], l0[k]);
            hi[k] = mx(hi[k], h0[k]);
        }
    }
    float ext = 0.0f;
    bool finite = true;
    for (int k = 0; k < 3; k++) {
        C.box[6 * (size_t)f + k] = lo[k];
        C.box[6 * (size_t)f + 3 + k] = hi[k];
        ext = fmaxf(ext, hi[k] - lo[k]);
    }
    const float xs[9] = {a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z};
    for (int k = 0; k < 9; k++) finite &= isfinite(xs[k]);
    if (!finite || !(ext < 3.0e38f)) {
        atomicOr(&C.ext[1], 1u);  // non-finite state: no cell size
        return;
    }
    atomicMax(&C.ext[0], __float_as_uint(ext));
}

__global__ void __launch_bounds__(128) cs_contact_node_kernel(Batch B, Contact C) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.N) return;
    v3 acc = mk3(0.0f, 0.0f, 0.0f);
    const v3 xi = ldx(B.x, i);
    for (int k = C.nf_ptr[i]; k < C.nf_ptr[i + 1]; k++) {
        const int code = C.nf_code[k];
        const int4 y = B.face_nodes[code >> 2];
        const int corner = code & 3;
        const int n1 = corner == 0 ? y.y : corner == 1 ? y.z : y.x;
        const int n2 = corner == 0 ? y.z : corner == 1 ? y.x : y.y;
        const v3 e0 = sub(ldx(B.x, n1), xi), e1 = sub(ldx(B.x, n2), xi);
        acc = add(acc, dvd(cross(e0, e1), dot0(e0, e0) * dot0(e1, e1)));
    }
    const v3 n = normalized(acc);
    C.nn[3 * (size_t)i] = n.x;
    C.nn[3 * (size_t)i + 1] = n.y;
    C.nn[3 * (size_t)i + 2] = n.z;
}

__global__ void __launch_bounds__(128) cs_contact_grid_kernel(Batch B, Contact C, const int* sheet_group) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= B.F || C.ext[1]) return;
    const float c = cell_size(C);
    const int group = sheet_group[B.face_nodes[f].w];
    int lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = cell_of(C.box[6 * (size_t)f + k], c);
        hi[k] = cell_of(C.box[6 * (size_t)f + 3 + k], c);
    }
    int slot = 0;
    for (int ix = lo[0]; ix <= hi[0]; ix++)
        for (int iy = lo[1]; iy <= hi[1]; iy++)
            for (int iz = lo[2]; iz <= hi[2]; iz++) {
                if (slot == 8) {
                    atomicOr(&C.ext[1], 2u);  // a face over more than 2 cells per axis
                    return;
                }
                const int e = 8 * f + slot++;
                C.next[e] = atomicExch(&C.head[bucket(C, group, ix, iy, iz)], e);
            }
}

// Candidate face pairs: thread per face f, walking the cells of its dilated bounds; each pair
// (f, g > f) of one collision group whose bounds overlap is appended once (in the lowest cell
// the two share).  Pairs are staged per thread and appended with one atomic per warp.
__global__ void __launch_bounds__(128) cs_contact_pair_kernel(Batch B, Contact C, const int* sheet_group) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    int2 buf[CS_PAIR_STAGE];
    int nb = 0;
    if (f < B.F && !C.ext[1]) {
        const float c = cell_size(C);
        const float t = C.dilate;  // 2 x repulsionThickness (Simulator.cu:274) or the collision thickness
        const int group = sheet_group[B.face_nodes[f].w];
        float dlo[3], dhi[3];
        int qlo[3], qhi[3];
        bool ok = true;
        for (int k = 0; k < 3; k++) {
            dlo[k] = C.box[6 * (size_t)f + k] - t;  // Bounds::dilate (Bounds.cu:60-68)
            dhi[k] = C.box[6 * (size_t)f + 3 + k] + t;
            qlo[k] = cell_of(dlo[k], c);
            qhi[k] = cell_of(dhi[k], c);
            ok &= qhi[k] - qlo[k] <= 2;
        }
        if (!ok) atomicOr(&C.ext[1], 4u);
        const long long walk_cap = 8LL * B.F + 8;
        for (int ix = qlo[0]; ok && ix <= qhi[0]; ix++)
            for (int iy = qlo[1]; ok && iy <= qhi[1]; iy++)
                for (int iz = qlo[2]; ok && iz <= qhi[2]; iz++) {
                    long long walked = 0;
                    for (int e = C.head[bucket(C, group, ix, iy, iz)]; e >= 0; e = C.next[e]) {
                        if (++walked > walk_cap) {
                            atomicOr(&C.ext[1], 8u);
                            ok = false;
                            break;
                        }
                        const int g = e >> 3;
                        if (g <= f) continue;
                        if (sheet_group[B.face_nodes[g].w] != group) continue;
                        const float* gb = C.box + 6 * (size_t)g;
                        // Bounds::overlap(b, thickness) (Bounds.cu:85-101): g against f dilated
                        if (gb[0] > dhi[0] || gb[3] < dlo[0] || gb[1] > dhi[1] || gb[4] < dlo[1] || gb[2] > dhi[2] ||
                            gb[5] < dlo[2])
                            continue;
                        // one test per pair: in the lowest cell both cover
                        if (max(qlo[0], cell_of(gb[0], c)) != ix || max(qlo[1], cell_of(gb[1], c)) != iy ||
                            max(qlo[2], cell_of(gb[2], c)) != iz)
                            continue;
                        if (nb == CS_PAIR_STAGE) {
                            const int base = atomicAdd(C.pair_count, nb);
                            for (int k = 0; k < nb; k++)
                                if (base + k < C.pair_cap) C.pairs[base + k] = buf[k];
                            nb = 0;
                        }
                        buf[nb++] = make_int2(f, g);
                    }
                }
    }
    // warp-aggregated append of the staged pairs
    const int lane = threadIdx.x & 31;
    int incl = nb;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    int base = 0;
    if (lane == 31 && incl > 0) base = atomicAdd(C.pair_count, incl);
    base = __shfl_sync(0xffffffffu, base, 31) + incl - nb;
    for (int k = 0; k < nb; k++)
        if (base + k < C.pair_cap) C.pairs[base + k] = buf[k];
}

// checkProximities (Simulator.cu:263-269), vertex-face part: thread per (pair, corner): the
// three corners of the first face against the second, then the reverse.
__global__ void __launch_bounds__(256) cs_contact_vf_kernel(Batch B, Contact C, int npairs) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6LL * npairs) return;
    const int p = (int)(t / 6), k = (int)(t % 6);
    const int2 pr = C.pairs[p];
    const int f = k < 3 ? pr.x : pr.y, g = k < 3 ? pr.y : pr.x;
    const int4 y = B.face_nodes[f];
    const int i = k % 3;
    check_vf(B, C, i == 0 ? y.x : i == 1 ? y.y : y.z, g);
}

// checkProximities, edge-edge part: thread per (pair, edge of the first face, edge of the second).
__global__ void __launch_bounds__(256) cs_contact_ee_kernel(Batch B, Contact C, int npairs) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 9LL * npairs) return;
    const int p = (int)(t / 9), k = (int)(t % 9);
    const int2 pr = C.pairs[p];
    const int4 fe = C.face_edges[pr.x], ge = C.face_edges[pr.y];
    const int i = k / 3, j = k % 3;
    check_ee(B, C, i == 0 ? fe.x : i == 1 ? fe.y : fe.z, j == 0 ? ge.x : j == 1 ? ge.y : ge.z);
}

namespace {
__device__ __forceinline__ bool admitted(const Contact& C, long long k, unsigned long long& v) {
    if (k >= C.n_keys) return false;
    v = C.keys[k];
    return v != ~0ULL && __uint_as_float((unsigned)(v >> 32)) < 2.0f * C.repulsion;  // Simulator.cu:287-295
}
}  // namespace

// Compaction, pass 1: admitted keys per block of CS_CONTACT_ITEMS (each thread 16 consecutive).
__global__ void __launch_bounds__(256) cs_contact_count_kernel(Contact C) {
    const long long base = (long long)blockIdx.x * CS_CONTACT_ITEMS + 16LL * threadIdx.x;
    int cnt = 0;
    unsigned long long v;
    for (int j = 0; j < 16; j++) cnt += admitted(C, base + j, v) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    __shared__ int ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int k = 0; k < 8; k++) s += ws[k];
        C.block_count[blockIdx.x] = s;
    }
}

// Pass 2 (one block): exclusive offsets of the blocks, and the total.
__global__ void __launch_bounds__(1024) cs_contact_scan_kernel(Contact C, int nblocks) {
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblocks; b0 += 1024) {
        const int b = b0 + threadIdx.x;
        const int v = b < nblocks ? C.block_count[b] : 0;
        int incl = v;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
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
        const int prefix = carry + (wid > 0 ? ws[wid - 1] : 0) + incl - v;
        if (b < nblocks) C.block_count[b] = prefix;
        __syncthreads();
        if (threadIdx.x == 0) carry += ws[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) *C.total = carry;
}

namespace {
// Proximity(node, face) (Proximity.cu:5-12) and Proximity(edge0, edge1) (Proximity.cu:14-21)
__device__ void make_record(const Batch& B, const Contact& C, long long k, unsigned long long v, cs_proximity_desc& r) {
    const int other = (int)(unsigned)v;
    for (int i = 0; i < 4; i++) {
        for (int e = 0; e < 3; e++) r.x[i][e] = r.v[i][e] = 0.0f;
        r.mass[i] = 0.0f;
    }
    r.free_mask = 0;  // every node is a batch node
    r.mu = C.friction;  // cloth nodes are free (Mesh.cu:349): the cloth friction
    const long long nodeKeys = 2LL * B.N, edgeKeys = 2LL * C.E;
    v3 n;
    float h;
    if (k < nodeKeys || k >= nodeKeys + edgeKeys) {
        const bool nodeKey = k < nodeKeys;
        const int node = nodeKey ? (int)(k >> 1) : other;
        const int face = nodeKey ? other : (int)((k - nodeKeys - edgeKeys) >> 1);
        const int4 y = B.face_nodes[face];
        r.nodes[0] = node;
        r.nodes[1] = y.x;
        r.nodes[2] = y.y;
        r.nodes[3] = y.z;
        r.stiffness = C.stiffness * mn(C.node_area[node], B.face_area[face]);
        signed_vf(ldx(B.x, node), ldx(B.x, y.x), ldx(B.x, y.y), ldx(B.x, y.z), n, r.w, h);
    } else {
        const int e0 = (int)((k - nodeKeys) >> 1), e1 = other;
        const int4 a = C.edges[e0], b = C.edges[e1];
        r.nodes[0] = a.x;
        r.nodes[1] = a.y;
        r.nodes[2] = b.x;
        r.nodes[3] = b.y;
        r.stiffness = C.stiffness * mn(C.edge_area[e0], C.edge_area[e1]);
        signed_ee(ldx(B.x, a.x), ldx(B.x, a.y), ldx(B.x, b.x), ldx(B.x, b.y), n, r.w, h);
    }
    if (h < 0.0f) n = neg(n);
    r.normal[0] = n.x;
    r.normal[1] = n.y;
    r.normal[2] = n.z;
}
}  // namespace

// Pass 3: each block writes its admitted keys' records at its offset, in key order.
__global__ void __launch_bounds__(256) cs_contact_write_kernel(Batch B, Contact C) {
    const long long base = (long long)blockIdx.x * CS_CONTACT_ITEMS + 16LL * threadIdx.x;
    unsigned long long v;
    int cnt = 0;
    for (int j = 0; j < 16; j++) cnt += admitted(C, base + j, v) ? 1 : 0;
    // block-wide exclusive scan of the per-thread counts
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    __shared__ int ws[8];
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    int before = 0;
    for (int k = 0; k < wid; k++) before += ws[k];
    int pos = C.block_count[blockIdx.x] + before + incl - cnt;
    for (int j = 0; j < 16; j++) {
        if (!admitted(C, base + j, v)) continue;
        if (pos < C.out_cap) {
            cs_proximity_desc r;
            make_record(B, C, base + j, v, r);
            C.out[pos] = r;
        }
        pos++;
    }
}
