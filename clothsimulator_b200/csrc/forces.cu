// Element kernels of the implicit step and the deterministic block assembly.
//
// Compiled with -fmad=false: every expression below follows the reference's FP32 operation
// order (PhysicsHelper.cu:264-353, Material.cu:91-156, Face.cu:109-132, Edge.cu:101-111,
// Cloth.cu:42-169) without fused multiply-adds, so the assembled system matches the
// reference's CPU assembly entry by entry.
//
// Kernels:
//   cs_face_kernel   one thread per face: normal, wind drag, stretching force, its 9x9
//                    contribution -dt^2 J to A and the face's right-hand-side terms.
//   cs_edge_kernel   one thread per interior edge: dihedral bending force, the rank-one
//                    Jacobian factors (dtheta, coefficient) and the edge's right-hand side.
//   cs_gather_kernel one warp per 32-row slice: every block (i, j) of A sums its
//                    contributors in the reference's order (mass, faces by index, edges by
//                    index, handles) from a precomputed per-topology list: no atomics, no
//                    sort, bit-reproducible.  Diagonal slots also produce b, the 3x3
//                    block-Jacobi inverse and the slice's ||b||^2.
#include "cs_internal.h"

namespace {

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 ld3(const float* p, int i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 scl(float s, f3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ f3 mulv(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
// Vector.cuh operator/ multiplies by the reciprocal.
__device__ __forceinline__ f3 dvd(f3 a, float s) {
    float inv = 1.0f / s;
    return mk(a.x * inv, a.y * inv, a.z * inv);
}
__device__ __forceinline__ float dot(f3 a, f3 b) {
    float s = a.x * b.x;
    s += a.y * b.y;
    s += a.z * b.z;
    return s;
}
__device__ __forceinline__ float nrm(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 normalized(f3 a) { return dvd(a, nrm(a)); }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// Transformation::applyToPoint (Transformation.cu:82-84) with Quaternion::rotate (Quaternion.cu:
// 76-78) in the reference's FP32 order: s p + t with
// rotate(p) = p (qs^2 - |qv|^2) + (2 qv)(qv . p) + (2 (qv x p)) qs.  T = {s, t (3), qs, qv (3)}.
__device__ __forceinline__ f3 transform_point(const float* T, f3 p) {
    const f3 qv = mk(T[5], T[6], T[7]);
    const float qs = T[4];
    const float n2 = qv.x * qv.x + qv.y * qv.y + qv.z * qv.z;
    const float d = qv.x * p.x + qv.y * p.y + qv.z * p.z;
    const f3 r = add(add(mulv(p, qs * qs - n2), mulv(scl(2.0f, qv), d)), mulv(scl(2.0f, cross(qv, p)), qs));
    return add(scl(T[0], r), mk(T[1], T[2], T[3]));
}
__device__ __forceinline__ float clampf_(float x, float a, float b) { return x < a ? a : (x > b ? b : x); }
__device__ __forceinline__ float maxf_(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minf_(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float absf_(float a) { return a < 0.0f ? -a : a; }

// 3x3 block-Jacobi inverse in double (adjugate / determinant), stored in float.
__device__ __forceinline__ void block_inverse(const float a[9], float* Pi) {
    const double m00 = a[0], m01 = a[1], m02 = a[2], m10 = a[3], m11 = a[4], m12 = a[5], m20 = a[6], m21 = a[7],
                 m22 = a[8];
    const double c00 = m11 * m22 - m12 * m21, c01 = m12 * m20 - m10 * m22, c02 = m10 * m21 - m11 * m20;
    const double det = m00 * c00 + m01 * c01 + m02 * c02;
    const double id = det != 0.0 ? 1.0 / det : 0.0;
    Pi[0] = (float)(c00 * id);
    Pi[1] = (float)((m02 * m21 - m01 * m22) * id);
    Pi[2] = (float)((m01 * m12 - m02 * m11) * id);
    Pi[3] = (float)(c01 * id);
    Pi[4] = (float)((m00 * m22 - m02 * m20) * id);
    Pi[5] = (float)((m02 * m10 - m00 * m12) * id);
    Pi[6] = (float)(c02 * id);
    Pi[7] = (float)((m01 * m20 - m00 * m21) * id);
    Pi[8] = (float)((m00 * m11 - m01 * m10) * id);
}

// A SELL panel slot (panel * 32 + lane) as a row-major 3x3 block.
__device__ __forceinline__ void load_slot(const float* A, int slot, float a[9]) {
    const float* pn = A + (size_t)(slot >> 5) * CS_PANEL_FLOATS;
    const int lane = slot & 31;
    for (int e = 0; e < 4; e++) a[e] = pn[4 * lane + e];
    for (int e = 0; e < 4; e++) a[4 + e] = pn[128 + 4 * lane + e];
    a[8] = pn[256 + lane];
}
__device__ __forceinline__ void store_slot(float* A, int slot, const float a[9]) {
    float* pn = A + (size_t)(slot >> 5) * CS_PANEL_FLOATS;
    const int lane = slot & 31;
    for (int e = 0; e < 4; e++) pn[4 * lane + e] = a[e];
    for (int e = 0; e < 4; e++) pn[128 + 4 * lane + e] = a[4 + e];
    pn[256 + lane] = a[8];
}

// Material::stretchingStiffness (Material.cu:91-124): trilinear lookup on the 30^3 table.
__device__ __forceinline__ float4 stretch_stiffness(const float4* __restrict__ T, float G00, float G01, float G11) {
    const float hi = (float)(CS_TABLE_N - 1) - 1e-6f;
    float x = (G00 + 0.25f) * (float)CS_TABLE_N;
    x = clampf_(x, 0.0f, hi);
    int xi = (int)x;
    x -= xi;
    float y = (G11 + 0.25f) * (float)CS_TABLE_N;
    y = clampf_(y, 0.0f, hi);
    int yi = (int)y;
    y -= yi;
    float z = absf_(G01) * (float)CS_TABLE_N;
    z = clampf_(z, 0.0f, hi);
    int zi = (int)z;
    z -= zi;
    float w[8];
    w[0] = (1.0f - x) * (1.0f - y) * (1.0f - z);
    w[1] = (1.0f - x) * (1.0f - y) * z;
    w[2] = (1.0f - x) * y * (1.0f - z);
    w[3] = (1.0f - x) * y * z;
    w[4] = x * (1.0f - y) * (1.0f - z);
    w[5] = x * (1.0f - y) * z;
    w[6] = x * y * (1.0f - z);
    w[7] = x * y * z;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int t = 0; t < 8; t++) {
        int i = t >> 2, j = (t >> 1) & 1, k = t & 1;
        float4 s = __ldg(&T[((xi + i) * CS_TABLE_N + (yi + j)) * CS_TABLE_N + (zi + k)]);
        a.x += s.x * w[t];
        a.y += s.y * w[t];
        a.z += s.z * w[t];
        a.w += s.w * w[t];
    }
    return a;
}

// Material::bendingStiffness (Material.cu:126-156).  bias is the side's bias weight after
// the fold and clamp of Material.cu:130-133, precomputed from the rest uv edge.
__device__ __forceinline__ float bend_stiffness(const float* __restrict__ samples, float length, float angle,
                                                float area, float bias) {
    float curv = length * angle / area;
    float alpha = 0.5f * curv;
    float biasWeight = bias;
    int biasId = (int)biasWeight;
    biasWeight -= biasId;
    float valueWeight = 0.2f * alpha;
    valueWeight = minf_(valueWeight, 4.0f - 1e-6f);
    int valueId = (int)valueWeight;
    valueId = valueId > 0 ? valueId : 0;
    valueWeight -= valueId;
    float w00 = (1.0f - biasWeight) * (1.0f - valueWeight);
    float w01 = (1.0f - biasWeight) * valueWeight;
    float w10 = biasWeight * (1.0f - valueWeight);
    float w11 = biasWeight * valueWeight;
    float ans = 0.0f;
    ans += samples[biasId * 5 + valueId] * w00;
    ans += samples[biasId * 5 + valueId + 1] * w01;
    ans += samples[(biasId + 1) * 5 + valueId] * w10;
    ans += samples[(biasId + 1) * 5 + valueId + 1] * w11;
    return maxf_(ans, 0.0f);
}

// One entry h(p, q) of the stretching Hessian (PhysicsHelper.cu:283-286) with the
// reference's expression order.  p = 3a + kp, q = 3b + kq; fu_p = fu[kp], fv_p = fv[kp],
// D0a = D(0, a), D1a = D(1, a) and likewise for q; same = (kp == kq).
__device__ __forceinline__ float stretch_h(float fu_p, float fv_p, float fu_q, float fv_q, float D0a, float D1a,
                                           float D0b, float D1b, float k0, float k1, float k2, float k3, float gu,
                                           float gv, bool same) {
    float fuu_p = D0a * fu_p, fvv_p = D1a * fv_p, fuv_p = 0.5f * (D0a * fv_p + D1a * fu_p);
    float fuu_q = D0b * fu_q, fvv_q = D1b * fv_q, fuv_q = 0.5f * (D0b * fv_q + D1b * fu_q);
    float guDuu = same ? (gu * D0a) * D0b : 0.0f;
    float gvDvv = same ? (gv * D1a) * D1b : 0.0f;
    float guDvv = same ? (gu * D1a) * D1b : 0.0f;
    float gvDuu = same ? (gv * D0a) * D0b : 0.0f;
    float h = k0 * (fuu_p * fuu_q + guDuu);
    h += k2 * (fvv_p * fvv_q + gvDvv);
    h += k1 * (fuu_p * fvv_q + guDvv + fvv_p * fuu_q + gvDuu);
    h += 2.0f * k3 * (fuv_p * fuv_q);
    return h;
}

}  // namespace

// Face record (CS_FACE_REC = 120 floats, 16-byte aligned pieces for the gather's vector
// loads): the face's 9x9 contribution to A, -dt*dt*J, as nine row-major 3x3 blocks (block
// (a, b) at 12 (3a + b), three zero floats after each), dt*(f + dt*J*v) of the stretching
// term for node a at 108 + 4a .. 108 + 4a + 2, and dt * wind force added to each node at
// 111, 115, 119.
//
// face_eval evaluates one face exactly as Face::update (normal), the wind loop of
// Cloth::addExternalForces and stretchingForce (PhysicsHelper.cu:264-291) do.  With
// rec != nullptr it writes the face record; with fo/Jo it writes f and J as stretchingForce
// returns them (the inspection path).
__device__ __forceinline__ void face_eval(const Batch& B, int f, float* __restrict__ rec, float* __restrict__ fo,
                                          float* __restrict__ Jo) {
    const DevParams& P = *B.params;
    const float dt = P.dt;
    const float s = -dt * dt;
    int4 fn = B.face_nodes[f];
    const SheetDesc& sh = B.sheets[fn.w];
    f3 x0 = ld3(B.x, fn.x), x1 = ld3(B.x, fn.y), x2 = ld3(B.x, fn.z);
    f3 v0 = ld3(B.v, fn.x), v1 = ld3(B.v, fn.y), v2 = ld3(B.v, fn.z);
    float area = B.face_area[f];
    float4 inv = B.face_inv[f];  // (00, 01, 10, 11)

    // Face::update (Face.cu:124-127): normal from the current positions.
    f3 e1 = sub(x1, x0), e2 = sub(x2, x0);
    f3 n = normalized(cross(e1, e2));

    // Wind drag (Cloth.cu:105-122), on the rest area of a free face.
    f3 avg = dvd(add(add(v0, v1), v2), 3.0f);
    f3 rel = sub(mk(sh.wind_v[0], sh.wind_v[1], sh.wind_v[2]), avg);
    float vn = dot(n, rel);
    f3 vt = sub(rel, scl(vn, n));
    f3 force = dvd(scl(area, add(scl(sh.wind_density * absf_(vn) * vn, n), scl(sh.wind_drag, vt))), 3.0f);
    f3 fw = scl(dt, force);

    // F = [x1 - x0, x2 - x0] * inverse (Face.cu:109-111), G = (F^T F - I) / 2
    float F[3][2];
    {
        float e1a[3] = {e1.x, e1.y, e1.z}, e2a[3] = {e2.x, e2.y, e2.z};
#pragma unroll
        for (int i = 0; i < 3; i++) {
            float s0 = e1a[i] * inv.x;
            s0 += e2a[i] * inv.z;
            float s1 = e1a[i] * inv.y;
            s1 += e2a[i] * inv.w;
            F[i][0] = s0;
            F[i][1] = s1;
        }
    }
    float FtF00 = F[0][0] * F[0][0], FtF01 = F[0][0] * F[0][1], FtF11 = F[0][1] * F[0][1];
    FtF00 += F[1][0] * F[1][0];
    FtF01 += F[1][0] * F[1][1];
    FtF11 += F[1][1] * F[1][1];
    FtF00 += F[2][0] * F[2][0];
    FtF01 += F[2][0] * F[2][1];
    FtF11 += F[2][1] * F[2][1];
    float G00 = 0.5f * (FtF00 - 1.0f), G01 = 0.5f * (FtF01 - 0.0f), G11 = 0.5f * (FtF11 - 1.0f);
    float4 k = stretch_stiffness(B.tables + (size_t)sh.table * CS_TABLE_ENTRIES, G00, G01, G11);
    const float gu = maxf_(G00, 0.0f), gv = maxf_(G11, 0.0f);
    // D = [-Y.row0 - Y.row1, Y.row0, Y.row1] as columns (PhysicsHelper.cu:268-271)
    const float D0[3] = {-inv.x - inv.z, inv.x, inv.z};
    const float D1[3] = {-inv.y - inv.w, inv.y, inv.w};
    const float fu[3] = {F[0][0], F[1][0], F[2][0]};
    const float fv[3] = {F[0][1], F[1][1], F[2][1]};
    const float vel[9] = {v0.x, v0.y, v0.z, v1.x, v1.y, v1.z, v2.x, v2.y, v2.z};
#pragma unroll
    for (int p = 0; p < 9; p++) {
        const int a = p / 3, kp = p % 3;
        const float fuu = D0[a] * fu[kp], fvv = D1[a] * fv[kp], fuv = 0.5f * (D0[a] * fv[kp] + D1[a] * fu[kp]);
        // grad with the expression order of PhysicsHelper.cu:282; f = -area * grad
        float g = k.x * G00 * fuu;
        g += k.z * G11 * fvv;
        g += k.y * (G00 * fvv + G11 * fuu);
        g += 2.0f * k.w * G01 * fuv;
        const float fp = -area * g;
        float jv = 0.0f;
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int b = q / 3, kq = q % 3;
            const float h = stretch_h(fu[kp], fv[kp], fu[kq], fv[kq], D0[a], D1[a], D0[b], D1[b], k.x, k.y, k.z, k.w,
                                      gu, gv, kp == kq);
            const float J = -area * h;
            jv += (dt * J) * vel[q];
            if (rec) rec[12 * (3 * a + b) + 3 * kp + kq] = s * J;  // block (a, b): three float4
            if (Jo) Jo[9 * p + q] = J;
        }
        if (rec) rec[108 + 4 * a + kp] = dt * (fp + jv);
        if (fo) fo[p] = fp;
    }
    if (rec) {
#pragma unroll
        for (int blk = 0; blk < 9; blk++) rec[12 * blk + 9] = rec[12 * blk + 10] = rec[12 * blk + 11] = 0.0f;
        rec[111] = fw.x;
        rec[115] = fw.y;
        rec[119] = fw.z;
    }
}

// One thread per face; the block's records are staged in shared memory (row stride 121 floats,
// conflict-free) and written out as one contiguous, coalesced range.
__global__ void __launch_bounds__(64) cs_face_kernel(Batch B) {
    constexpr int kStride = CS_FACE_REC + 1;
    __shared__ float stage[64 * kStride];
    const int f0 = blockIdx.x * blockDim.x;
    const int f = f0 + threadIdx.x;
    if (f < B.F) face_eval(B, f, stage + threadIdx.x * kStride, nullptr, nullptr);
    __syncthreads();
    const int nf = min((int)blockDim.x, B.F - f0);
    float* out = B.face_rec + (size_t)f0 * CS_FACE_REC;
    for (int e = threadIdx.x; e < nf * CS_FACE_REC; e += blockDim.x)
        out[e] = stage[(e / CS_FACE_REC) * kStride + e % CS_FACE_REC];
}

// Edge record (32 floats): node i's (dtheta_i, coefficient) at [4i .. 4i + 3], dt*(f + dt*J*v)
// of the bending term for node i at [16 + 4i .. 16 + 4i + 2], theta at [19].
__global__ void __launch_bounds__(128) cs_edge_kernel(Batch B) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= B.E) return;
    const DevParams& P = *B.params;
    const float dt = P.dt;
    int4 en = B.edge_nodes[e];
    int meta = B.edge_meta[e];
    const SheetDesc& sh = B.sheets[B.edge_sheet[e]];
    float4 par = B.edge_par[e];
    f3 x0 = ld3(B.x, en.x), x1 = ld3(B.x, en.y), x2 = ld3(B.x, en.z), x3 = ld3(B.x, en.w);

    // Adjacent face normals with each face's own vertex order (Face.cu:124-127).
    // Face 0's cyclic vertex order is a rotation of (x0, x1, opposite0), face 1's of
    // (x1, x0, opposite1); meta holds the two rotations.
    f3 n0, n1;
    {
        int r = meta & 3;
        f3 a = r == 0 ? x0 : (r == 1 ? x1 : x2);
        f3 b = r == 0 ? x1 : (r == 1 ? x2 : x0);
        f3 c = r == 0 ? x2 : (r == 1 ? x0 : x1);
        n0 = normalized(cross(sub(b, a), sub(c, a)));
        r = (meta >> 2) & 3;
        a = r == 0 ? x1 : (r == 1 ? x0 : x3);
        b = r == 0 ? x0 : (r == 1 ? x3 : x1);
        c = r == 0 ? x3 : (r == 1 ? x1 : x0);
        n1 = normalized(cross(sub(b, a), sub(c, a)));
    }
    // bendingForce (PhysicsHelper.cu:327-353)
    float length = nrm(sub(x1, x0));
    float angle;
    {
        f3 ee = normalized(sub(x0, x1));
        float sine = dot(ee, cross(n0, n1));
        float cosine = dot(n0, n1);
        angle = (float)atan2((double)sine, (double)cosine);
    }
    float area = par.x;
    f3 ed = sub(x1, x0);
    float en2 = dot(ed, ed);
    float h0, h1, w00, w01, w10, w11;
    {
        f3 t = sub(x2, x0);
        f3 rr = dvd(mulv(ed, dot(ed, t)), en2);
        h0 = nrm(sub(t, rr));
        float tt = dot(ed, sub(x2, x0)) / en2;
        w00 = 1.0f - tt;
        w01 = tt;
    }
    {
        f3 t = sub(x3, x0);
        f3 rr = dvd(mulv(ed, dot(ed, t)), en2);
        h1 = nrm(sub(t, rr));
        float tt = dot(ed, sub(x3, x0)) / en2;
        w10 = 1.0f - tt;
        w11 = tt;
    }
    f3 a0 = sub(dvd(scl(-w00, n0), h0), dvd(scl(w10, n1), h1));
    f3 a1 = sub(dvd(scl(-w01, n0), h0), dvd(scl(w11, n1), h1));
    f3 a2 = dvd(n0, h0);
    f3 a3 = dvd(n1, h1);
    float dth[12] = {a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, a2.x, a2.y, a2.z, a3.x, a3.y, a3.z};
    float k0 = bend_stiffness(sh.bending, length, angle, area, par.y);
    float k1 = bend_stiffness(sh.bending, length, angle, area, par.z);
    float coef = -0.25f * minf_(k0, k1) * (length * length) / area;
    float ca = coef * angle;

    f3 v0 = ld3(B.v, en.x), v1 = ld3(B.v, en.y), v2 = ld3(B.v, en.z), v3 = ld3(B.v, en.w);
    float vel[12] = {v0.x, v0.y, v0.z, v1.x, v1.y, v1.z, v2.x, v2.y, v2.z, v3.x, v3.y, v3.z};
    float bb[12];
#pragma unroll
    for (int p = 0; p < 12; p++) {
        float jv = 0.0f;
#pragma unroll
        for (int q = 0; q < 12; q++) jv += (dt * (coef * (dth[p] * dth[q]))) * vel[q];
        bb[p] = dt * (ca * dth[p] + jv);
    }
    float4* out = reinterpret_cast<float4*>(B.edge_rec + (size_t)e * CS_EDGE_REC);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        out[i] = make_float4(dth[3 * i], dth[3 * i + 1], dth[3 * i + 2], coef);
        out[4 + i] = make_float4(bb[3 * i], bb[3 * i + 1], bb[3 * i + 2], i == 0 ? angle : 0.0f);
    }
}

// Assembly gather.  Warps walk the slices grid-stride (a persistent launch of a few warps per
// SM), so the slices in flight at any moment cover a few sheets and their element records
// stay in L2.  Lane = row.  For every block slot the contributors are summed in the
// reference's order; their codes and record values are fetched four at a time so several
// loads are in flight before the ordered additions.  Writes A's panels, and for the
// diagonal slot b, the block-Jacobi inverse and the slice's ||b||^2 (part[2*slice]).
__global__ void __launch_bounds__(128) cs_gather_kernel(Batch B) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const DevParams& P = *B.params;
    const float dt = P.dt;
    const float s = -dt * dt;
    for (int slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; slice < B.n_slices; slice += warps) {
        const SliceDesc sd = B.slices[slice];
        const SheetDesc& sh = B.sheets[sd.sheet];
        const bool live = lane < sd.rows;
        const int row = sd.row0 + (live ? B.rowmap[sd.topo_slice * CS_SLICE + lane] : 0);
        const float* __restrict__ frec = B.face_rec + (size_t)sh.face_off * CS_FACE_REC;
        const float* __restrict__ erec = B.edge_rec + (size_t)sh.edge_off * CS_EDGE_REC;
        double bsq = 0.0;
        for (int k = 0; k < sd.width; k++) {
            const int tslot = (sd.tpanel0 + k) * CS_SLICE + lane;
            float a[9];
#pragma unroll
            for (int t = 0; t < 9; t++) a[t] = 0.0f;
            int c0 = 0, c1 = 0;
            if (live) {
                if (k == 0) {
                    const float m = B.mass[row];
                    a[0] = m; a[4] = m; a[8] = m;
                }
                c0 = __ldg(&B.tcptr[tslot]);
                c1 = __ldg(&B.tcptr[tslot + 1]);
                for (int c = c0; c < c1; c += 4) {
                    uint32_t code[4];
                    float v[4][9];
#pragma unroll
                    for (int j = 0; j < 4; j++) code[j] = (c + j < c1) ? __ldg(&B.tcontrib[c + j]) : 0u;
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        if (c + j >= c1) continue;
                        const int elem = (int)((code[j] >> 4) & 0x7FFFFFFu);
                        const int ca = (code[j] >> 2) & 3, cb = code[j] & 3;
                        if (!(code[j] & CS_CODE_EDGE)) {
                            const float4* r = reinterpret_cast<const float4*>(frec + (size_t)elem * CS_FACE_REC +
                                                                              12 * (3 * ca + cb));
                            const float4 q0 = __ldg(r), q1 = __ldg(r + 1), q2 = __ldg(r + 2);
                            v[j][0] = q0.x; v[j][1] = q0.y; v[j][2] = q0.z; v[j][3] = q0.w;
                            v[j][4] = q1.x; v[j][5] = q1.y; v[j][6] = q1.z; v[j][7] = q1.w;
                            v[j][8] = q2.x;
                        } else {
                            const float4* r = reinterpret_cast<const float4*>(erec + (size_t)elem * CS_EDGE_REC);
                            const float4 qa = __ldg(r + ca), qb = __ldg(r + cb);
                            const float coef = qa.w;
                            const float da[3] = {qa.x, qa.y, qa.z}, db[3] = {qb.x, qb.y, qb.z};
#pragma unroll
                            for (int kk = 0; kk < 3; kk++)
#pragma unroll
                                for (int hh = 0; hh < 3; hh++) v[j][3 * kk + hh] = s * (coef * (da[kk] * db[hh]));
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (c + j < c1)
#pragma unroll
                            for (int e = 0; e < 9; e++) a[e] += v[j][e];
                }
                if (k == 0) {
                    const int hc = (int)B.handle[row].w;
                    for (int t = 0; t < hc; t++) {
                        const float add_ = dt * dt * P.handle_stiffness;
                        a[0] += add_; a[4] += add_; a[8] += add_;
                    }
                }
            }
            // streaming stores: A is read back from DRAM by the solvers, while the element
            // records this kernel re-reads should keep their place in L2
            float* panel = B.A + (size_t)(sd.panel0 + k) * CS_PANEL_FLOATS;
            __stcs(reinterpret_cast<float4*>(panel) + lane, make_float4(a[0], a[1], a[2], a[3]));
            __stcs(reinterpret_cast<float4*>(panel + 128) + lane, make_float4(a[4], a[5], a[6], a[7]));
            __stcs(panel + 256 + lane, a[8]);

            if (k == 0 && live) {
                // Right-hand side in the reference's order: gravity, wind (faces), stretching
                // (faces), bending (edges), handles (Cloth.cu:94-169).
                const float m = B.mass[row];
                const float g0 = (dt * m) * P.gravity[0], g1 = (dt * m) * P.gravity[1], g2 = (dt * m) * P.gravity[2];
                float b0 = 0.0f + g0, b1 = 0.0f + g1, b2 = 0.0f + g2;
                for (int pass = 0; pass < 3; pass++) {
                    for (int c = c0; c < c1; c += 4) {
                        float w[4][3];
                        bool use[4];
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            use[j] = false;
                            if (c + j >= c1) continue;
                            const uint32_t code = __ldg(&B.tcontrib[c + j]);
                            const bool edge = (code & CS_CODE_EDGE) != 0;
                            if (edge != (pass == 2)) continue;
                            const int elem = (int)((code >> 4) & 0x7FFFFFFu);
                            const int ca = (code >> 2) & 3;
                            if (pass == 0) {
                                const float* r = frec + (size_t)elem * CS_FACE_REC;
                                w[j][0] = __ldg(r + 111);
                                w[j][1] = __ldg(r + 115);
                                w[j][2] = __ldg(r + 119);
                            } else {
                                const float4 q = __ldg(reinterpret_cast<const float4*>(
                                    pass == 1 ? frec + (size_t)elem * CS_FACE_REC + 108 + 4 * ca
                                              : erec + (size_t)elem * CS_EDGE_REC + 16 + 4 * ca));
                                w[j][0] = q.x;
                                w[j][1] = q.y;
                                w[j][2] = q.z;
                            }
                            use[j] = true;
                        }
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            if (use[j]) {
                                b0 += w[j][0];
                                b1 += w[j][1];
                                b2 += w[j][2];
                            }
                    }
                }
                const float4 hd = B.handle[row];
                const int hc = (int)hd.w;
                if (hc > 0) {
                    const f3 xr = ld3(B.x, row), vr = ld3(B.v, row);
                    // the target: the handle's position at load, or a motion's transformation of it
                    const int mo = B.handle_motion[row];
                    const f3 target = mo >= 0 ? transform_point(B.params->motion[mo], mk(hd.x, hd.y, hd.z))
                                              : mk(hd.x, hd.y, hd.z);
                    const f3 fh = mulv(scl(dt, sub(sub(target, xr), scl(dt, vr))), P.handle_stiffness);
                    for (int t = 0; t < hc; t++) {
                        b0 += fh.x; b1 += fh.y; b2 += fh.z;
                    }
                }
                B.b[3 * row] = b0;
                B.b[3 * row + 1] = b1;
                B.b[3 * row + 2] = b2;
                bsq = (double)b0 * b0 + (double)b1 * b1 + (double)b2 * b2;
                block_inverse(a, B.Pinv + 9 * (size_t)row);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bsq += __shfl_xor_sync(0xffffffffu, bsq, o);
        if (lane == 0) B.part[2 * slice] = bsq;
    }
}

// The reference's per-element outputs (f, J) for inspection: faces re-evaluated from the
// current state as stretchingForce returns them (PhysicsHelper.cu:288-290), interior edges
// expanded from the last assembly's records as bendingForce returns them
// (PhysicsHelper.cu:351-352).
__global__ void __launch_bounds__(128) cs_expand_kernel(Batch B, float* face_f, float* face_J, float* edge_f,
                                                        float* edge_J) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < B.F) face_eval(B, i, nullptr, face_f + 9 * (size_t)i, face_J + 81 * (size_t)i);
    if (i < B.E) {
        const float* r = B.edge_rec + (size_t)i * CS_EDGE_REC;
        const float coef = r[3], angle = r[19];
        const float ca = coef * angle;
        float d[12];
        for (int p = 0; p < 12; p++) d[p] = r[4 * (p / 3) + p % 3];
        for (int p = 0; p < 12; p++) {
            edge_f[12 * (size_t)i + p] = ca * d[p];
            for (int q = 0; q < 12; q++) edge_J[144 * (size_t)i + 12 * p + q] = coef * (d[p] * d[q]);
        }
    }
}

// ---------------------------------------------------------------------------------------
// Proximity terms (Cloth::addProximityForces, Cloth.cu:171-192), one thread per (proximity,
// sheet) instance: penetration depth below the thickness, the impulse and friction forces
// and Jacobians of impulseForce / frictionForce (PhysicsHelper.cu:398-432) in FP32 with the
// reference's operation order (this file is built without FMA contraction), written as the
// element blocks -dt^2 J_imp, -dt J_fr and right-hand sides dt (f_imp + dt J_imp v), dt f_fr.
__global__ void __launch_bounds__(128) cs_prox_kernel(Batch B) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= B.n_pinst) return;
    const ProxInst& P = B.pinst[t];
    const float dt = B.params->dt;
    const float th = P.thickness;
    f3 xs[4], vs[4];
    float ms[4];
    int freeMask = 0;
    for (int i = 0; i < 4; i++) {
        const int nd = P.node[i];
        if (nd >= 0) {
            xs[i] = ld3(B.x, nd);
            vs[i] = ld3(B.v, nd);
            ms[i] = B.mass[nd];
            freeMask |= 1 << i;  // cloth nodes are free (Mesh.cu:349)
        } else {
            xs[i] = mk(P.xe[i][0], P.xe[i][1], P.xe[i][2]);
            vs[i] = mk(P.ve[i][0], P.ve[i][1], P.ve[i][2]);
            ms[i] = P.me[i];
            if ((P.free_mask >> i) & 1) freeMask |= 1 << i;
        }
    }
    const f3 n = mk(P.n[0], P.n[1], P.n[2]);
    // d = max(h - sum_i w_i n.x_i, 0) (Cloth.cu:179-182)
    float d = -th;
    for (int i = 0; i < 4; i++) d += P.w[i] * dot(n, xs[i]);
    d = maxf_(-d, 0.0f);
    float* rec = B.prec + (size_t)t * CS_PROX_REC;
    // impulseForce: f = 1/2 k/h d^2 N, J = -k/h d N N^T
    float N[12], vel[12];
    for (int i = 0; i < 4; i++) {
        N[3 * i] = P.w[i] * n.x;
        N[3 * i + 1] = P.w[i] * n.y;
        N[3 * i + 2] = P.w[i] * n.z;
        vel[3 * i] = vs[i].x;
        vel[3 * i + 1] = vs[i].y;
        vel[3 * i + 2] = vs[i].z;
    }
    const float sf = 0.5f * P.stiffness / th * (d * d);
    const float sj = -P.stiffness / th * d;
    const float s2 = -dt * dt;
    for (int p = 0; p < 12; p++) {
        float jv = 0.0f;
        for (int q = 0; q < 12; q++) {
            const float J = sj * (N[p] * N[q]);
            rec[12 * p + q] = s2 * J;
            jv += (dt * J) * vel[q];
        }
        rec[288 + p] = dt * (sf * N[p] + jv);
    }
    // frictionForce: F = 1/2 k/h d^2; vt = (I - n n^T) sum_i w_i v_i;
    // f_v = min(mu F / |vt|, 1 / (dt sum_free w_i^2 / m_i)); f = -f_v (w_i vt);
    // J_ij = -f_v w_i w_j (I - n n^T)
    const float F = 0.5f * P.stiffness / th * (d * d);
    f3 v = mk(0.0f, 0.0f, 0.0f);
    float invMass = 0.0f;
    for (int i = 0; i < 4; i++) {
        v = add(v, scl(P.w[i], vs[i]));
        if ((freeMask >> i) & 1) invMass += (P.w[i] * P.w[i]) / ms[i];
    }
    float T[3][3];
    const float nn[3] = {n.x, n.y, n.z};
    for (int k = 0; k < 3; k++)
        for (int h = 0; h < 3; h++) T[k][h] = (k == h ? 1.0f : 0.0f) - nn[k] * nn[h];
    const float vv[3] = {v.x, v.y, v.z};
    float vt[3];
    for (int k = 0; k < 3; k++) {
        float acc = 0.0f;
        for (int h = 0; h < 3; h++) acc += T[k][h] * vv[h];
        vt[k] = acc;
    }
    const float vtn = sqrtf(0.0f + vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]);
    const float f_v = minf_(P.mu * F / vtn, 1.0f / (dt * invMass));
    const float s1 = -dt;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            const float s = -f_v * P.w[i] * P.w[j];
            for (int k = 0; k < 3; k++)
                for (int h = 0; h < 3; h++) rec[144 + (3 * i + k) * 12 + 3 * j + h] = s1 * (s * T[k][h]);
        }
    for (int i = 0; i < 4; i++)
        for (int c = 0; c < 3; c++) rec[300 + 3 * i + c] = dt * (-f_v * (P.w[i] * vt[c]));
}

// Proximity terms onto the system, one thread per row holding a proximity node, in the order
// Cloth::addProximityForces accumulates them (Cloth.cu:171-192 through addElement's coeffRef,
// Cloth.cu:42-76): instances ascending, impulse before friction, row corner, column corner;
// after the gather's handle terms.  Blocks on the mesh pattern are summed onto their slot,
// others onto the row's side list (zeroed first); the row's block-Jacobi inverse is redone.
__global__ void __launch_bounds__(128) cs_prox_row_kernel(Batch B) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= B.N) return;
    const int q0 = B.prow_ptr[row], q1 = B.prow_ptr[row + 1];
    if (q0 == q1) return;
    const SheetDesc& sd = B.sheets[B.node_sheet[row]];
    const int* cp = B.tcsr_ptr + sd.csr_ptr_off;
    const int li = row - sd.node_off;
    const int c0 = cp[li], c1 = cp[li + 1];
    // SELL slot of block (row, col) on the mesh pattern, or -1
    auto slot_of = [&](int col) {
        const int lj = col - sd.node_off;
        int lo = c0, hi = c1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (B.tcsr_col[mid] < lj) lo = mid + 1;
            else hi = mid;
        }
        return (lo < c1 && B.tcsr_col[lo] == lj) ? sd.panel_off * CS_SLICE + B.tcsr_slot[lo] : -1;
    };
    const int x0 = B.xptr ? B.xptr[row] : 0, x1 = B.xptr ? B.xptr[row + 1] : 0;
    for (int m = x0; m < x1; m++)
        for (int e = 0; e < 9; e++) B.xval[9 * (size_t)m + e] = 0.0f;
    float b0 = B.b[3 * row], b1 = B.b[3 * row + 1], b2 = B.b[3 * row + 2];
    for (int q = q0; q < q1; q++) {
        const int inst = B.prow_inst[q];
        const ProxInst& P = B.pinst[inst];
        const float* rec = B.prec + (size_t)inst * CS_PROX_REC;
        for (int fr = 0; fr < 2; fr++)
            for (int a = 0; a < 4; a++) {
                if (!((P.local >> a) & 1) || P.node[a] != row) continue;
                const float* r = rec + (fr ? 300 : 288) + 3 * a;
                b0 += r[0];
                b1 += r[1];
                b2 += r[2];
                for (int bb = 0; bb < 4; bb++) {
                    if (!((P.local >> bb) & 1)) continue;
                    const int col = P.node[bb];
                    const float* blk = rec + fr * 144 + (3 * a) * 12 + 3 * bb;
                    const int slot = slot_of(col);
                    float acc[9];
                    float* dst = nullptr;
                    if (slot >= 0) {
                        load_slot(B.A, slot, acc);
                    } else {
                        int m = x0;
                        while (m < x1 && B.xcol[m] != col) m++;
                        if (m == x1) continue;  // not listed: cannot happen for a consistent list
                        dst = B.xval + 9 * (size_t)m;
                        for (int e = 0; e < 9; e++) acc[e] = dst[e];
                    }
                    for (int k = 0; k < 3; k++)
                        for (int h = 0; h < 3; h++) acc[3 * k + h] += blk[k * 12 + h];
                    if (slot >= 0) store_slot(B.A, slot, acc);
                    else
                        for (int e = 0; e < 9; e++) dst[e] = acc[e];
                }
            }
    }
    B.b[3 * row] = b0;
    B.b[3 * row + 1] = b1;
    B.b[3 * row + 2] = b2;
    const int ds = slot_of(row);
    if (ds >= 0) {
        float a[9];
        load_slot(B.A, ds, a);
        block_inverse(a, B.Pinv + 9 * (size_t)row);
    }
}

// ||b||^2 per slice after the proximity right-hand sides (the gather's partials otherwise).
__global__ void __launch_bounds__(128) cs_slice_bnorm_kernel(Batch B) {
    const int slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (slice >= B.n_slices) return;
    const SliceDesc sd = B.slices[slice];
    double bsq = 0.0;
    if (lane < sd.rows) {
        const int row = sd.row0 + B.rowmap[sd.topo_slice * CS_SLICE + lane];
        const float b0 = B.b[3 * row], b1 = B.b[3 * row + 1], b2 = B.b[3 * row + 2];
        bsq = (double)b0 * b0 + (double)b1 * b1 + (double)b2 * b2;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bsq += __shfl_xor_sync(0xffffffffu, bsq, o);
    if (lane == 0) B.part[2 * slice] = bsq;
}
