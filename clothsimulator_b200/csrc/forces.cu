// Element kernels of the implicit step and the deterministic block assembly.
//
// Compiled with -fmad=false: every expression below follows the reference's FP32 operation
// order (PhysicsHelper.cu:264-353, Material.cu:91-156, Face.cu:109-132, Edge.cu:101-111,
// Cloth.cu:42-169) without fused multiply-adds, so the assembled system matches the
// reference's CPU assembly entry by entry.
//
// Kernels:
//   cs_edge_kernel   one thread per interior edge: dihedral bending geometry (dtheta, the
//                    rank-one Jacobian's coefficient, theta) as a 64-byte record.
//   cs_gather_kernel one warp per 32-row slice, lane = row: the row's own rows of the
//                    stretching terms of its faces (evaluated here) and of the bending terms of
//                    its interior edges, summed into every block (i, j) of A in the reference's
//                    order (mass, faces by index, edges by index, handles) in shared memory: no
//                    atomics, no sort, bit-reproducible.  Also b, the 3x3 block-Jacobi inverse
//                    and the slice's ||b||^2.
//   cs_expand_kernel the per-element f and J as the reference's force functions return them
//                    (inspection).
//   cs_prox_kernel, cs_prox_row_kernel  proximity terms on top of the assembled system.
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

namespace {

// One face's stretching terms: the state its rows share (stretchingForce's set-up,
// PhysicsHelper.cu:264-281, with F from Face.cu:109-111), then one row p = 3a + kp at a time.
struct FaceState {
    float area;
    float G00, G01, G11, gu, gv;
    float4 k;
    float D0[3], D1[3], fu[3], fv[3], vel[9];
};

__device__ __forceinline__ void face_setup(const Batch& B, int f, FaceState& S) {
    const int4 fn = B.face_nodes[f];
    const SheetDesc& sh = B.sheets[fn.w];
    const f3 x0 = ld3(B.x, fn.x), x1 = ld3(B.x, fn.y), x2 = ld3(B.x, fn.z);
    const f3 v0 = ld3(B.v, fn.x), v1 = ld3(B.v, fn.y), v2 = ld3(B.v, fn.z);
    S.area = B.face_area[f];
    const float4 inv = B.face_inv[f];  // (00, 01, 10, 11)
    const f3 e1 = sub(x1, x0), e2 = sub(x2, x0);
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
    S.G00 = 0.5f * (FtF00 - 1.0f);
    S.G01 = 0.5f * (FtF01 - 0.0f);
    S.G11 = 0.5f * (FtF11 - 1.0f);
    S.k = stretch_stiffness(B.tables + (size_t)sh.table * CS_TABLE_ENTRIES, S.G00, S.G01, S.G11);
    S.gu = maxf_(S.G00, 0.0f);
    S.gv = maxf_(S.G11, 0.0f);
    // D = [-Y.row0 - Y.row1, Y.row0, Y.row1] as columns (PhysicsHelper.cu:268-271)
    S.D0[0] = -inv.x - inv.z;
    S.D0[1] = inv.x;
    S.D0[2] = inv.z;
    S.D1[0] = -inv.y - inv.w;
    S.D1[1] = inv.y;
    S.D1[2] = inv.w;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        S.fu[i] = F[i][0];
        S.fv[i] = F[i][1];
    }
    const float vel[9] = {v0.x, v0.y, v0.z, v1.x, v1.y, v1.z, v2.x, v2.y, v2.z};
#pragma unroll
    for (int i = 0; i < 9; i++) S.vel[i] = vel[i];
}

// Row p = 3a + kp of the face's stretching terms: f_p (returned in fp) and, for each column
// q, J(p, q) handed to emit(q, J) in column order; returns dt (f_p + dt sum_q J(p, q) v_q), the
// row's right-hand-side term, with the reference's operation order (PhysicsHelper.cu:282-290).
template <class Emit>
__device__ __forceinline__ float face_row(const FaceState& S, int p, float dt, float& fp, Emit emit) {
    const int a = p / 3, kp = p % 3;
    // the row's corner and component by selects (no indexed local arrays)
    const float D0a = a == 0 ? S.D0[0] : (a == 1 ? S.D0[1] : S.D0[2]);
    const float D1a = a == 0 ? S.D1[0] : (a == 1 ? S.D1[1] : S.D1[2]);
    const float fup = kp == 0 ? S.fu[0] : (kp == 1 ? S.fu[1] : S.fu[2]);
    const float fvp = kp == 0 ? S.fv[0] : (kp == 1 ? S.fv[1] : S.fv[2]);
    const float fuu = D0a * fup, fvv = D1a * fvp, fuv = 0.5f * (D0a * fvp + D1a * fup);
    // grad with the expression order of PhysicsHelper.cu:282; f = -area * grad
    float g = S.k.x * S.G00 * fuu;
    g += S.k.z * S.G11 * fvv;
    g += S.k.y * (S.G00 * fvv + S.G11 * fuu);
    g += 2.0f * S.k.w * S.G01 * fuv;
    fp = -S.area * g;
    float jv = 0.0f;
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const int b = q / 3, kq = q % 3;
        const float h = stretch_h(fup, fvp, S.fu[kq], S.fv[kq], D0a, D1a, S.D0[b], S.D1[b], S.k.x, S.k.y, S.k.z, S.k.w, S.gu,
                                  S.gv, kp == kq);
        const float J = -S.area * h;
        jv += (dt * J) * S.vel[q];
        emit(q, J);
    }
    return dt * (fp + jv);
}

// dt times the wind drag on each node of a face (Cloth.cu:105-122) on its rest area, from the
// normal of the current positions (Face::update, Face.cu:124-127).
__device__ __forceinline__ f3 face_wind(const Batch& B, int f, float dt) {
    const int4 fn = B.face_nodes[f];
    const SheetDesc& sh = B.sheets[fn.w];
    const f3 x0 = ld3(B.x, fn.x), x1 = ld3(B.x, fn.y), x2 = ld3(B.x, fn.z);
    const f3 v0 = ld3(B.v, fn.x), v1 = ld3(B.v, fn.y), v2 = ld3(B.v, fn.z);
    const float area = B.face_area[f];
    const f3 n = normalized(cross(sub(x1, x0), sub(x2, x0)));
    const f3 avg = dvd(add(add(v0, v1), v2), 3.0f);
    const f3 rel = sub(mk(sh.wind_v[0], sh.wind_v[1], sh.wind_v[2]), avg);
    const float vn = dot(n, rel);
    const f3 vt = sub(rel, scl(vn, n));
    const f3 force = dvd(scl(area, add(scl(sh.wind_density * absf_(vn) * vn, n), scl(sh.wind_drag, vt))), 3.0f);
    return scl(dt, force);
}

// Dihedral bending of one interior edge (bendingForce, PhysicsHelper.cu:327-353, with the
// adjacent face normals of Face.cu:124-127 and the bending stiffness of Material.cu:126-156):
// the gradient dtheta (4 nodes x 3), the coefficient of the rank-one Jacobian
// coef dtheta dtheta^T and the angle theta; f = coef theta dtheta.
__device__ __forceinline__ void edge_geom(const Batch& B, int e, float (&dth)[12], float& coef, float& angle) {
    const int4 en = B.edge_nodes[e];
    const int meta = B.edge_meta[e];
    const SheetDesc& sh = B.sheets[B.edge_sheet[e]];
    const float4 par = B.edge_par[e];
    const f3 x0 = ld3(B.x, en.x), x1 = ld3(B.x, en.y), x2 = ld3(B.x, en.z), x3 = ld3(B.x, en.w);
    // Adjacent face normals with each face's own vertex order (Face.cu:124-127).  Face 0's
    // cyclic vertex order is a rotation of (x0, x1, opposite0), face 1's of (x1, x0,
    // opposite1); meta holds the two rotations.
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
    const float length = nrm(sub(x1, x0));
    {
        f3 ee = normalized(sub(x0, x1));
        float sine = dot(ee, cross(n0, n1));
        float cosine = dot(n0, n1);
        angle = (float)atan2((double)sine, (double)cosine);
    }
    const float area = par.x;
    const f3 ed = sub(x1, x0);
    const float en2 = dot(ed, ed);
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
    const f3 a0 = sub(dvd(scl(-w00, n0), h0), dvd(scl(w10, n1), h1));
    const f3 a1 = sub(dvd(scl(-w01, n0), h0), dvd(scl(w11, n1), h1));
    const f3 a2 = dvd(n0, h0);
    const f3 a3 = dvd(n1, h1);
    const float d[12] = {a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, a2.x, a2.y, a2.z, a3.x, a3.y, a3.z};
#pragma unroll
    for (int i = 0; i < 12; i++) dth[i] = d[i];
    const float k0 = bend_stiffness(sh.bending, length, angle, area, par.y);
    const float k1 = bend_stiffness(sh.bending, length, angle, area, par.z);
    coef = -0.25f * minf_(k0, k1) * (length * length) / area;
}

}  // namespace

// One thread per interior edge: its bending geometry (edge_geom) once, as a 64-byte record
// {dtheta 0-2, coef}, {dtheta 3-5, theta}, {dtheta 6-8, 0}, {dtheta 9-11, 0} that the
// gather's four rows of the edge read (the records of the slices in flight stay in L2).
__global__ void __launch_bounds__(128) cs_edge_kernel(Batch B) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= B.E) return;
    float d[12], coef, angle;
    edge_geom(B, e, d, coef, angle);
    float4* out = B.edge_geo + 4 * (size_t)e;
    out[0] = make_float4(d[0], d[1], d[2], coef);
    out[1] = make_float4(d[3], d[4], d[5], angle);
    out[2] = make_float4(d[6], d[7], d[8], 0.0f);
    out[3] = make_float4(d[9], d[10], d[11], 0.0f);
}

// Assembly.  Warps walk the slices grid-stride (a persistent launch); lane = row.  Each row
// evaluates its own rows of the stretching terms of its faces (face_row, shared with the
// inspection kernel below) and forms its rows of the bending terms of its interior edges from
// their records (cs_edge_kernel), and adds each block into the row's slot accumulators in
// shared memory:
// faces in index order, then edges in index order, after the mass and before the handles, so
// every block (i, j) sums its contributors in the reference's order (Cloth.cu:78-169) with no
// atomics.  b follows the reference's order too: gravity, wind (faces), stretching (faces),
// bending (edges), handles (Cloth.cu:94-169).  A face is evaluated by each of its three
// corner rows (a third of its rows each); face records, nine 3x3 blocks per face, would be
// read back through L2 by rows far apart in the slice order.  Writes A's panels, b, the block-Jacobi inverse
// of the diagonal block and the slice's ||b||^2 (part[2*slice]).
//
// Dynamic shared memory: per warp gather_width slots x 9 entries x 32 lanes, entry e of slot k
// of a lane at [(9 k + e) * 32 + lane] (each lane touches only its own words: no conflicts).
// Row lists (per topology node, at its sheet's row2slot_off): rface = {face << 2 | corner,
// the row's slots of the face's corners 0..2, 8 bits each}, redge likewise for the interior
// edges' corners 0..3.
extern __shared__ float cs_gather_acc[];

__global__ void __launch_bounds__(CS_GATHER_THREADS) cs_gather_kernel(Batch B) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const DevParams& P = *B.params;
    const float dt = P.dt;
    const float s = -dt * dt;
    float* const acc = cs_gather_acc + (size_t)(threadIdx.x >> 5) * B.gather_width * 9 * CS_SLICE + lane;
    for (int slice = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; slice < B.n_slices; slice += warps) {
        const SliceDesc sd = B.slices[slice];
        const SheetDesc& sh = B.sheets[sd.sheet];
        const bool live = lane < sd.rows;
        const int lrow = live ? B.rowmap[sd.topo_slice * CS_SLICE + lane] : 0;
        const int row = sd.row0 + lrow;
        const float m = live ? B.mass[row] : 0.0f;
        for (int k = 0; k < sd.width; k++)
#pragma unroll
            for (int e = 0; e < 9; e++) acc[(9 * k + e) * CS_SLICE] = (k == 0 && (e & 3) == 0) ? m : 0.0f;
        float b0 = 0.0f, b1 = 0.0f, b2 = 0.0f;
        if (live) {
            const int base = sh.row2slot_off + lrow;
            const int f0 = __ldg(&B.rface_ptr[base]), f1 = __ldg(&B.rface_ptr[base + 1]);
            const int e0 = __ldg(&B.redge_ptr[base]), e1 = __ldg(&B.redge_ptr[base + 1]);
            b0 += (dt * m) * P.gravity[0];
            b1 += (dt * m) * P.gravity[1];
            b2 += (dt * m) * P.gravity[2];
            for (int t = f0; t < f1; t++) {
                const f3 w = face_wind(B, sh.face_off + (__ldg(&B.rface[t].x) >> 2), dt);
                b0 += w.x;
                b1 += w.y;
                b2 += w.z;
            }
            for (int t = f0; t < f1; t++) {
                const int2 c = __ldg(&B.rface[t]);
                FaceState S;
                face_setup(B, sh.face_off + (c.x >> 2), S);
                const int a = c.x & 3;
                float r[3];
#pragma unroll
                for (int kp = 0; kp < 3; kp++) {
                    float fp;
                    r[kp] = face_row(S, 3 * a + kp, dt, fp, [&](int q, float J) {
                        acc[(9 * ((c.y >> (8 * (q / 3))) & 0xff) + 3 * kp + q % 3) * CS_SLICE] += s * J;
                    });
                }
                b0 += r[0];
                b1 += r[1];
                b2 += r[2];
            }
            for (int t = e0; t < e1; t++) {
                const int2 c = __ldg(&B.redge[t]);
                const int e = sh.edge_off + (c.x >> 2), a = c.x & 3;
                float dth[12], coef, angle;
                {
                    const float4* rec = B.edge_geo + 4 * (size_t)e;
                    const float4 q0 = __ldg(rec), q1 = __ldg(rec + 1), q2 = __ldg(rec + 2), q3 = __ldg(rec + 3);
                    dth[0] = q0.x; dth[1] = q0.y; dth[2] = q0.z; coef = q0.w;
                    dth[3] = q1.x; dth[4] = q1.y; dth[5] = q1.z; angle = q1.w;
                    dth[6] = q2.x; dth[7] = q2.y; dth[8] = q2.z;
                    dth[9] = q3.x; dth[10] = q3.y; dth[11] = q3.z;
                }
                // the row's node's gradient by selects (no indexed local arrays)
                float da[3];
#pragma unroll
                for (int kk = 0; kk < 3; kk++)
                    da[kk] = a == 0 ? dth[kk] : (a == 1 ? dth[3 + kk] : (a == 2 ? dth[6 + kk] : dth[9 + kk]));
                // the row's rank-one blocks (a, b), b = 0..3, onto their slots
#pragma unroll
                for (int bb = 0; bb < 4; bb++) {
                    float* d = acc + 9 * ((c.y >> (8 * bb)) & 0xff) * CS_SLICE;
#pragma unroll
                    for (int kk = 0; kk < 3; kk++)
#pragma unroll
                        for (int hh = 0; hh < 3; hh++) d[(3 * kk + hh) * CS_SLICE] += s * (coef * (da[kk] * dth[3 * bb + hh]));
                }
                // dt (f + dt J v) of the row's node (PhysicsHelper.cu:351-352)
                const int4 en = B.edge_nodes[e];
                const f3 v0 = ld3(B.v, en.x), v1 = ld3(B.v, en.y), v2 = ld3(B.v, en.z), v3 = ld3(B.v, en.w);
                const float vel[12] = {v0.x, v0.y, v0.z, v1.x, v1.y, v1.z, v2.x, v2.y, v2.z, v3.x, v3.y, v3.z};
                const float ca = coef * angle;
                float r[3];
#pragma unroll
                for (int kk = 0; kk < 3; kk++) {
                    float jv = 0.0f;
#pragma unroll
                    for (int q = 0; q < 12; q++) jv += (dt * (coef * (da[kk] * dth[q]))) * vel[q];
                    r[kk] = dt * (ca * da[kk] + jv);
                }
                b0 += r[0];
                b1 += r[1];
                b2 += r[2];
            }
            const float4 hd = B.handle[row];
            const int hc = (int)hd.w;
            if (hc > 0) {
                const float add_ = dt * dt * P.handle_stiffness;
                for (int t = 0; t < hc; t++) {
                    acc[0] += add_;
                    acc[4 * CS_SLICE] += add_;
                    acc[8 * CS_SLICE] += add_;
                }
                const f3 xr = ld3(B.x, row), vr = ld3(B.v, row);
                // the target: the handle's position at load, or a motion's transformation of it
                const int mo = B.handle_motion[row];
                const f3 target = mo >= 0 ? transform_point(B.params->motion[mo], mk(hd.x, hd.y, hd.z))
                                          : mk(hd.x, hd.y, hd.z);
                const f3 fh = mulv(scl(dt, sub(sub(target, xr), scl(dt, vr))), P.handle_stiffness);
                for (int t = 0; t < hc; t++) {
                    b0 += fh.x;
                    b1 += fh.y;
                    b2 += fh.z;
                }
            }
        }
        // the panels, streamed (the solvers read A back from DRAM)
        double bsq = 0.0;
        for (int k = 0; k < sd.width; k++) {
            float a[9];
#pragma unroll
            for (int e = 0; e < 9; e++) a[e] = acc[(9 * k + e) * CS_SLICE];
            float* panel = B.A + (size_t)(sd.panel0 + k) * CS_PANEL_FLOATS;
            __stcs(reinterpret_cast<float4*>(panel) + lane, make_float4(a[0], a[1], a[2], a[3]));
            __stcs(reinterpret_cast<float4*>(panel + 128) + lane, make_float4(a[4], a[5], a[6], a[7]));
            __stcs(panel + 256 + lane, a[8]);
            if (k == 0 && live) {
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

// The reference's per-element outputs (f, J) for inspection, from the current state: faces
// as stretchingForce returns them (PhysicsHelper.cu:288-290), interior edges as bendingForce
// returns them (PhysicsHelper.cu:351-352).
__global__ void __launch_bounds__(128) cs_expand_kernel(Batch B, float* face_f, float* face_J, float* edge_f,
                                                        float* edge_J) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float dt = B.params->dt;
    if (i < B.F) {
        FaceState S;
        face_setup(B, i, S);
        float* Jo = face_J + 81 * (size_t)i;
        for (int p = 0; p < 9; p++) {
            float fp;
            face_row(S, p, dt, fp, [&](int q, float J) { Jo[9 * p + q] = J; });
            face_f[9 * (size_t)i + p] = fp;
        }
    }
    if (i < B.E) {
        float d[12], coef, angle;
        edge_geom(B, i, d, coef, angle);
        const float ca = coef * angle;
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
