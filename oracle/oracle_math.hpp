// CPU restatement of ClothSimulator's per-element physics, for use as a TEST ORACLE ONLY.
//
// Nothing in the product library includes this file; only the oracle shared library
// (oracle/oracle.cpp), the reference adapter (oracle/ref_adapter.cu), tests and the
// CPU-baseline leg of bench.py reach it.  Every function restates a reference
// function and cites it.  With T = float the operation order follows the reference
// expression by expression so that, compiled without FMA contraction, the results
// are the reference's FP32 results; with T = double the same code is the FP64 oracle.
#ifndef CLOTHSTEP_ORACLE_MATH_HPP
#define CLOTHSTEP_ORACLE_MATH_HPP

#include <cmath>
#include <cstdint>

namespace orc {

constexpr int kTableN = 30;  // Material.cuh:16 (const int N = 30)

template <class T> struct V2 { T a[2]; T& operator[](int i) { return a[i]; } const T& operator[](int i) const { return a[i]; } };
template <class T> struct V3 { T a[3]; T& operator[](int i) { return a[i]; } const T& operator[](int i) const { return a[i]; } };

template <class T> inline V3<T> v3(T x, T y, T z) { return V3<T>{{x, y, z}}; }
template <class T> inline V3<T> sub(const V3<T>& p, const V3<T>& q) { return v3(p[0] - q[0], p[1] - q[1], p[2] - q[2]); }
template <class T> inline V3<T> add(const V3<T>& p, const V3<T>& q) { return v3(p[0] + q[0], p[1] + q[1], p[2] + q[2]); }
template <class T> inline V3<T> scl(T s, const V3<T>& p) { return v3(s * p[0], s * p[1], s * p[2]); }
template <class T> inline V3<T> mul(const V3<T>& p, T s) { return v3(p[0] * s, p[1] * s, p[2] * s); }
// Vector.cuh operator/: multiplies by the reciprocal (Vector.cuh:128-134).
template <class T> inline V3<T> dvd(const V3<T>& p, T s) { T inv = T(1) / s; return v3(p[0] * inv, p[1] * inv, p[2] * inv); }
template <class T> inline T dot(const V3<T>& p, const V3<T>& q) { T s = T(0); s += p[0] * q[0]; s += p[1] * q[1]; s += p[2] * q[2]; return s; }
template <class T> inline T norm2(const V3<T>& p) { return dot(p, p); }
template <class T> inline T norm(const V3<T>& p) { return std::sqrt(norm2(p)); }
template <class T> inline V3<T> normalized(const V3<T>& p) { return dvd(p, norm(p)); }
// Vector.cuh:173-176
template <class T> inline V3<T> cross(const V3<T>& p, const V3<T>& q) {
    return v3(p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]);
}
template <class T> inline T mn(T a, T b) { return a < b ? a : b; }   // MathHelper.cuh:15
template <class T> inline T mx(T a, T b) { return a > b ? a : b; }   // MathHelper.cuh:19
template <class T> inline T ab(T x) { return x < T(0) ? -x : x; }    // MathHelper.cuh:23
template <class T> inline T clampv(T x, T a, T b) { return x < a ? a : (x > b ? b : x); }  // MathHelper.cuh:27

// Real-type specific library calls: the FP32 reference calls the float overloads.
inline float r_atan2(float y, float x) { return std::atan2(y, x); }
inline double r_atan2(double y, double x) { return std::atan2(y, x); }

// 2x2 symmetric eigen-decomposition, MathHelper.cu:3-36.
template <class T>
inline void eigen2(T a, T b, T d, T Q[2][2], T l[2]) {
    T amd = a - d;
    T apd = a + d;
    T b2 = b * b;
    T det = std::sqrt(T(4) * b2 + amd * amd);
    T l1 = T(0.5) * (apd + det);
    T l2 = T(0.5) * (apd - det);
    l[0] = l1;
    l[1] = l2;
    if (b != T(0)) {
        T v0 = l1 - d, v1 = b;
        T vn = std::sqrt(v0 * v0 + b2);
        Q[0][0] = v0 / vn;
        Q[1][0] = v1 / vn;
        v0 = l2 - d;
        vn = std::sqrt(v0 * v0 + b2);
        Q[0][1] = v0 / vn;
        Q[1][1] = v1 / vn;
    } else if (a >= d) {
        Q[0][0] = T(1); Q[1][0] = T(0); Q[0][1] = T(0); Q[1][1] = T(1);
    } else {
        Q[0][0] = T(0); Q[1][0] = T(1); Q[0][1] = T(1); Q[1][1] = T(0);
    }
}

// Data-driven material (Wang et al. 2011 table), Material.cu:3-156.
template <class T>
struct Material {
    T density;
    T samples[kTableN][kTableN][kTableN][4];
    T bending[3][5];

    // Material.cu:45-85 (calculateStretchingSample).  `data` is the 2x5 grid of 4-vectors
    // built at Material.cu:20-27.
    static void sample(T G00, T G01, T G11, const T data[2][5][4], T out[4]) {
        T Q[2][2], l[2];
        eigen2<T>(T(2) * G00, T(2) * G01, T(2) * G11, Q, l);
        if (l[0] == l[1] && Q[0][0] == T(0) && Q[1][1] == T(0)) {
            Q[0][0] = T(1); Q[0][1] = T(0); Q[1][0] = T(0); Q[1][1] = T(1);
        }
        if (Q[0][0] < T(0)) { Q[0][0] = -Q[0][0]; Q[1][0] = -Q[1][0]; }
        if (Q[1][1] < T(0)) { Q[0][1] = -Q[0][1]; Q[1][1] = -Q[1][1]; }

        T strainWeight = (std::sqrt(l[0] + T(1)) - T(1)) * T(6);
        strainWeight = clampv<T>(strainWeight, T(0), T(1) - T(1e-6f));
        int strainId = static_cast<int>(strainWeight);
        strainWeight -= strainId;

        // abs(atan2(..)) / M_PI * 8.0f: the division by the double constant M_PI is
        // evaluated in double precision before the result is stored as T.
        T angleWeight = static_cast<T>(static_cast<double>(ab(r_atan2(Q[1][0], Q[0][0]))) / M_PI * 8.0f);
        angleWeight = clampv<T>(angleWeight, T(0), T(4) - T(1e-6f));
        int angleId = static_cast<int>(angleWeight);
        angleWeight -= angleId;

        T w[2][2];
        w[0][0] = (T(1) - strainWeight) * (T(1) - angleWeight);
        w[0][1] = (T(1) - strainWeight) * angleWeight;
        w[1][0] = strainWeight * (T(1) - angleWeight);
        w[1][1] = strainWeight * angleWeight;
        T ans[4] = {T(0), T(0), T(0), T(0)};
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++)
                for (int c = 0; c < 4; c++) ans[c] += data[strainId + i][angleId + j][c] * w[i][j];
        for (int c = 0; c < 4; c++) out[c] = mx<T>(ans[c], T(0)) * T(2);
    }

    // Material.cu:3-41.  stretching6x4: the file's six rows; bending3x5: the file's samples.
    void build(T file_density, const T stretching6x4[6][4], const T bending3x5[3][5], T thicken, T density_mult,
               T stretching_mult, T bending_mult) {
        T densityMultiplier = density_mult * thicken;
        T stretchingMultiplier = stretching_mult * thicken;
        T bendingMultiplier = bending_mult * thicken;
        density = file_density * densityMultiplier;
        T data[2][5][4];
        for (int c = 0; c < 4; c++) data[0][0][c] = stretching6x4[0][c];
        for (int i = 1; i < 5; i++)
            for (int c = 0; c < 4; c++) data[0][i][c] = data[0][0][c];
        for (int i = 0; i < 5; i++)
            for (int c = 0; c < 4; c++) data[1][i][c] = stretching6x4[i + 1][c];
        for (int i = 0; i < kTableN; i++)
            for (int j = 0; j < kTableN; j++)
                for (int k = 0; k < kTableN; k++) {
                    T G00 = static_cast<T>(static_cast<float>(i) / kTableN - 0.25f);
                    T G11 = static_cast<T>(static_cast<float>(j) / kTableN - 0.25f);
                    T G01 = static_cast<T>(static_cast<float>(k) / kTableN);
                    T s[4];
                    sample(G00, G01, G11, data, s);
                    for (int c = 0; c < 4; c++) samples[i][j][k][c] = s[c] * stretchingMultiplier;
                }
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 5; j++) bending[i][j] = bending3x5[i][j] * bendingMultiplier;
    }

    // Material.cu:91-124 (trilinear lookup over G00, G11, |G01|).
    void stretchingStiffness(T G00, T G01, T G11, T out[4]) const {
        const T hi = T(kTableN - 1) - T(1e-6f);
        T x = (G00 + T(0.25f)) * T(kTableN);
        x = clampv<T>(x, T(0), hi);
        int xi = static_cast<int>(x);
        x -= xi;
        T y = (G11 + T(0.25f)) * T(kTableN);
        y = clampv<T>(y, T(0), hi);
        int yi = static_cast<int>(y);
        y -= yi;
        T z = ab(G01) * T(kTableN);
        z = clampv<T>(z, T(0), hi);
        int zi = static_cast<int>(z);
        z -= zi;
        T w[2][2][2];
        w[0][0][0] = (T(1) - x) * (T(1) - y) * (T(1) - z);
        w[0][0][1] = (T(1) - x) * (T(1) - y) * z;
        w[0][1][0] = (T(1) - x) * y * (T(1) - z);
        w[0][1][1] = (T(1) - x) * y * z;
        w[1][0][0] = x * (T(1) - y) * (T(1) - z);
        w[1][0][1] = x * (T(1) - y) * z;
        w[1][1][0] = x * y * (T(1) - z);
        w[1][1][1] = x * y * z;
        for (int c = 0; c < 4; c++) out[c] = T(0);
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++)
                for (int k = 0; k < 2; k++)
                    for (int c = 0; c < 4; c++) out[c] += samples[xi + i][yi + j][zi + k][c] * w[i][j][k];
    }

    // Material.cu:126-156.
    T bendingStiffness(T length, T angle, T area, T d0, T d1) const {
        T curv = length * angle / area;
        T alpha = T(0.5f) * curv;
        T biasWeight = static_cast<T>(static_cast<double>(ab(r_atan2(d1, d0)) * T(4)) / M_PI);
        if (biasWeight > T(2)) biasWeight = T(4) - biasWeight;
        biasWeight = clampv<T>(biasWeight, T(0), T(2) - T(1e-6f));
        int biasId = static_cast<int>(biasWeight);
        biasWeight -= biasId;
        T valueWeight = T(0.2f) * alpha;
        valueWeight = mn<T>(valueWeight, T(4) - T(1e-6f));
        int valueId = static_cast<int>(valueWeight);
        valueId = valueId > 0 ? valueId : 0;
        valueWeight -= valueId;
        T w[2][2];
        w[0][0] = (T(1) - biasWeight) * (T(1) - valueWeight);
        w[0][1] = (T(1) - biasWeight) * valueWeight;
        w[1][0] = biasWeight * (T(1) - valueWeight);
        w[1][1] = biasWeight * valueWeight;
        T ans = T(0);
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) ans += bending[biasId + i][valueId + j] * w[i][j];
        return mx<T>(ans, T(0));
    }
};

// Face rest data, Face.cu:12-20: inverse of [u1-u0, u2-u0] (Matrix.cuh:184-197) and rest area.
template <class T>
inline void faceRest(const T u0[2], const T u1[2], const T u2[2], T inv[2][2], T& area) {
    T d1[2] = {u1[0] - u0[0], u1[1] - u0[1]};
    T d2[2] = {u2[0] - u0[0], u2[1] - u0[1]};
    // Matrix2x2f(d1, d2) holds d1, d2 as columns.
    T a = d1[0], b = d2[0], c = d1[1], d = d2[1];
    T invDet = T(1) / (a * d - b * c);
    inv[0][0] = d * invDet;
    inv[0][1] = -b * invDet;
    inv[1][0] = -c * invDet;
    inv[1][1] = a * invDet;
    T cr = d1[0] * d2[1] - d1[1] * d2[0];
    area = T(0.5f) * ab(cr);
}

// Face normal, Face.cu:124-127.
template <class T>
inline V3<T> faceNormal(const V3<T>& x0, const V3<T>& x1, const V3<T>& x2) {
    return normalized(cross(sub(x1, x0), sub(x2, x0)));
}

// Membrane stretching force and Jacobian of one face, PhysicsHelper.cu:264-291.
// J is row-major 9x9, f has 9 entries (node-major, xyz).
template <class T>
inline void stretchingForce(const Material<T>& mat, const V3<T>& x0, const V3<T>& x1, const V3<T>& x2,
                            const T inv[2][2], T area, T f[9], T J[81]) {
    V3<T> e1 = sub(x1, x0), e2 = sub(x2, x0);
    // F = Matrix3x2f(e1, e2) * inverse  (Face.cu:109-111)
    T F[3][2];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 2; j++) {
            T s = T(0);
            s += e1[i] * inv[0][j];
            s += e2[i] * inv[1][j];
            F[i][j] = s;
        }
    // G = 0.5 (F^T F - I)
    T FtF[2][2];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            T s = T(0);
            for (int k = 0; k < 3; k++) s += F[k][i] * F[k][j];
            FtF[i][j] = s;
        }
    T G[2][2];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) G[i][j] = T(0.5f) * (FtF[i][j] - (i == j ? T(1) : T(0)));

    // D = [-Y.row0 - Y.row1, Y.row0, Y.row1] as columns.
    T D[2][3];
    D[0][0] = -inv[0][0] - inv[1][0];
    D[1][0] = -inv[0][1] - inv[1][1];
    D[0][1] = inv[0][0];
    D[1][1] = inv[0][1];
    D[0][2] = inv[1][0];
    D[1][2] = inv[1][1];

    T fu[3] = {F[0][0], F[1][0], F[2][0]};
    T fv[3] = {F[0][1], F[1][1], F[2][1]};
    T fuu[9], fvv[9], fuv[9];
    for (int a = 0; a < 3; a++)
        for (int k = 0; k < 3; k++) {
            fuu[3 * a + k] = D[0][a] * fu[k];
            fvv[3 * a + k] = D[1][a] * fv[k];
            fuv[3 * a + k] = T(0.5f) * (D[0][a] * fv[k] + D[1][a] * fu[k]);
        }
    T k[4];
    mat.stretchingStiffness(G[0][0], G[0][1], G[1][1], k);

    T grad[9];
    for (int p = 0; p < 9; p++) {
        T g = k[0] * G[0][0] * fuu[p];
        g += k[2] * G[1][1] * fvv[p];
        g += k[1] * (G[0][0] * fvv[p] + G[1][1] * fuu[p]);
        g += T(2) * k[3] * G[0][1] * fuv[p];
        grad[p] = g;
    }
    T gu = mx<T>(G[0][0], T(0)), gv = mx<T>(G[1][1], T(0));
    for (int p = 0; p < 9; p++) {
        int a = p / 3, kp = p % 3;
        for (int q = 0; q < 9; q++) {
            int b = q / 3, kq = q % 3;
            // max(G,0) * D^T * D evaluates as ((g * D^T) * D): one non-zero product per entry.
            bool same = (kp == kq);
            T guDuu = same ? (gu * D[0][a]) * D[0][b] : T(0);
            T gvDvv = same ? (gv * D[1][a]) * D[1][b] : T(0);
            T guDvv = same ? (gu * D[1][a]) * D[1][b] : T(0);
            T gvDuu = same ? (gv * D[0][a]) * D[0][b] : T(0);
            T h = k[0] * (fuu[p] * fuu[q] + guDuu);
            h += k[2] * (fvv[p] * fvv[q] + gvDvv);
            h += k[1] * (fuu[p] * fvv[q] + guDvv + fvv[p] * fuu[q] + gvDuu);
            h += T(2) * k[3] * (fuv[p] * fuv[q]);
            J[9 * p + q] = -area * h;
        }
        f[p] = -area * grad[p];
    }
}

// PhysicsHelper.cu:314-319
template <class T>
inline T pointLineDistance(const V3<T>& x, const V3<T>& a, const V3<T>& b) {
    V3<T> e = sub(b, a);
    V3<T> t = sub(x, a);
    V3<T> r = dvd(mul(e, dot(e, t)), norm2(e));
    return norm(sub(t, r));
}

// PhysicsHelper.cu:321-325
template <class T>
inline void barycentric(const V3<T>& x, const V3<T>& a, const V3<T>& b, T w[2]) {
    V3<T> e = sub(b, a);
    T t = dot(e, sub(x, a)) / norm2(e);
    w[0] = T(1) - t;
    w[1] = t;
}

// Dihedral angle of an interior edge, Edge.cu:101-111.
template <class T>
inline T edgeAngle(const V3<T>& xa, const V3<T>& xb, const V3<T>& n0, const V3<T>& n1) {
    V3<T> e = normalized(sub(xa, xb));
    T sine = dot(e, cross(n0, n1));
    T cosine = dot(n0, n1);
    return r_atan2(sine, cosine);
}

// Bending force and Gauss-Newton Jacobian of one interior edge, PhysicsHelper.cu:327-353.
// x0, x1: the edge's nodes; x2, x3: the opposite nodes of adjacent faces 0 and 1;
// n0, n1: those faces' normals; area: sum of their rest areas; d0, d1: uv edge vectors
// (vertices[s][1].u - vertices[s][0].u) of the two sides.  J is row-major 12x12.
template <class T>
inline void bendingForce(const Material<T>& mat, const V3<T>& x0, const V3<T>& x1, const V3<T>& x2, const V3<T>& x3,
                         const V3<T>& n0, const V3<T>& n1, T area, const T d0[2], const T d1[2], T f[12], T J[144],
                         T* theta_out = nullptr) {
    T length = norm(sub(x1, x0));
    T angle = edgeAngle(x0, x1, n0, n1);
    T h0 = pointLineDistance(x2, x0, x1);
    T h1 = pointLineDistance(x3, x0, x1);
    T w0[2], w1[2];
    barycentric(x2, x0, x1, w0);
    barycentric(x3, x0, x1, w1);
    V3<T> a0 = sub(dvd(scl(-w0[0], n0), h0), dvd(scl(w1[0], n1), h1));
    V3<T> a1 = sub(dvd(scl(-w0[1], n0), h0), dvd(scl(w1[1], n1), h1));
    V3<T> a2 = dvd(n0, h0);
    V3<T> a3 = dvd(n1, h1);
    T dtheta[12];
    for (int c = 0; c < 3; c++) {
        dtheta[c] = a0[c];
        dtheta[3 + c] = a1[c];
        dtheta[6 + c] = a2[c];
        dtheta[9 + c] = a3[c];
    }
    T k0 = mat.bendingStiffness(length, angle, area, d0[0], d0[1]);
    T k1 = mat.bendingStiffness(length, angle, area, d1[0], d1[1]);
    T coefficient = T(-0.25f) * mn<T>(k0, k1) * (length * length) / area;
    T ca = coefficient * angle;
    for (int p = 0; p < 12; p++) {
        f[p] = ca * dtheta[p];
        for (int q = 0; q < 12; q++) J[12 * p + q] = coefficient * (dtheta[p] * dtheta[q]);
    }
    if (theta_out) *theta_out = angle;
}

// ---------------------------------------------------------------------------------------
// Proximity forces (the repulsion and friction terms of Cloth::physicsStep,
// Cloth.cu:171-192).  A proximity (Proximity.cuh:11-21) couples four nodes through weights
// w (vertex-face: 1 and minus the barycentric weights; edge-edge: the edge weights), a unit
// normal n, a friction coefficient mu and a stiffness already scaled by the smaller area
// (Proximity.cu:7-24).

// impulseForce (PhysicsHelper.cu:398-406): f = 1/2 k/h d^2 N, J = -k/h d N N^T with
// N = (w_0 n, w_1 n, w_2 n, w_3 n).
template <class T>
inline void impulseForce(const T w[4], const V3<T>& n, T stiffness, T d, T thickness, T f[12], T J[144]) {
    T N[12];
    for (int i = 0; i < 4; i++)
        for (int c = 0; c < 3; c++) N[3 * i + c] = w[i] * n[c];
    const T sf = T(0.5) * stiffness / thickness * (d * d);
    for (int p = 0; p < 12; p++) f[p] = sf * N[p];
    const T sj = -stiffness / thickness * d;
    for (int p = 0; p < 12; p++)
        for (int q = 0; q < 12; q++) J[12 * p + q] = sj * (N[p] * N[q]);
}

// frictionForce (PhysicsHelper.cu:408-432): tangential relative velocity vt of the weighted
// nodes, magnitude f_v = min(mu F / |vt|, 1 / (dt sum_free w_i^2 / m_i)), f = -f_v (w_i vt),
// J_ij = -f_v w_i w_j (I - n n^T).
template <class T>
inline void frictionForce(const T w[4], const V3<T>& n, T mu, T stiffness, T d, T thickness, T dt, const V3<T> vel[4],
                          const T mass[4], int freeMask, T f[12], T J[144]) {
    const T F = T(0.5) * stiffness / thickness * (d * d);
    V3<T> v = v3(T(0), T(0), T(0));
    T invMass = T(0);
    for (int i = 0; i < 4; i++) {
        V3<T> wv = scl(w[i], vel[i]);
        v = add(v, wv);
        if (freeMask & (1 << i)) invMass += (w[i] * w[i]) / mass[i];
    }
    T Tm[3][3];
    for (int k = 0; k < 3; k++)
        for (int h = 0; h < 3; h++) Tm[k][h] = (k == h ? T(1) : T(0)) - n[k] * n[h];
    V3<T> vt;
    for (int k = 0; k < 3; k++) {
        T acc = T(0);
        for (int h = 0; h < 3; h++) acc += Tm[k][h] * v[h];
        vt[k] = acc;
    }
    const T f_v = mn(mu * F / norm(vt), T(1) / (dt * invMass));
    for (int i = 0; i < 4; i++)
        for (int c = 0; c < 3; c++) f[3 * i + c] = -f_v * (w[i] * vt[c]);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            const T s = -f_v * w[i] * w[j];
            for (int k = 0; k < 3; k++)
                for (int h = 0; h < 3; h++) J[(3 * i + k) * 12 + 3 * j + h] = s * Tm[k][h];
        }
}

// Penetration depth below the thickness (Cloth.cu:179-182): d = max(h - sum_i w_i n.x_i, 0).
template <class T>
inline T proximityDepth(const T w[4], const V3<T>& n, const V3<T> x[4], T thickness) {
    T d = -thickness;
    for (int i = 0; i < 4; i++) d += w[i] * dot(n, x[i]);
    return mx(-d, T(0));
}

}  // namespace orc

#endif
