// The collision step restated for the CPU oracle.  TEST INFRASTRUCTURE ONLY: nothing in the
// product library includes this file.
//
// Restates Simulator::collisionStep as its GPU path runs it (Simulator.cu:602-684, the
// `gpu` branch: every round tests all candidate pairs, without the CPU branch's BVH
// activity flags): continuous impacts between the positions at the start of the step (x0)
// and the current ones (checkImpact, CollisionHelper.cu:61-110, with solveCubic, solveQuadratic
// and newtonsMethod, :3-59), over face pairs whose x0-and-x bounds overlap after dilating one
// by the collision thickness (BVH with ccd bounds, Face::bounds, Face.cu:94-103), the
// per-element bounds checks of checkVertexFaceImpact / checkEdgeEdgeImpact (:112-136), the
// selection of independent impacts by impact time (Simulator.cu:394-420), the impact-zone
// projection CollisionOptimization (CollisionOptimization.cu:5-145) solved by the augmented
// Lagrangian gradient descent of Optimization::solve (Optimization.cu:94-137, constants
// Optimization.cuh:15-18), up to MAX_COLLISION_ITERATION = 100 rounds per deformation level
// (CollisionHelper.cuh:21), and the velocity update v = (x - x0) / dt (Mesh.cu:238-247).
// All cloth nodes are free (no obstacles), so the two deformation levels behave alike.
// Impacts with equal times are ordered by their node ids (the reference's sort leaves them
// in traversal order).
#ifndef CLOTHSTEP_ORACLE_COLLIDE_HPP
#define CLOTHSTEP_ORACLE_COLLIDE_HPP

#include <algorithm>
#include <cmath>
#include <functional>
#include <vector>

#include "oracle_detect.hpp"
#include "oracle_math.hpp"

namespace orc {

constexpr int kMaxCollisionRounds = 100;   // CollisionHelper.cuh:21
constexpr int kMaxOptIterations = 100;     // Optimization.cuh:15
constexpr float kEpsS = 1e-12f;            // Optimization.cuh:16
constexpr float kEpsF = 1e-10f;            // Optimization.cuh:17

struct Impact {
    int type;      // 0 vertex-face, 1 edge-edge
    int nodes[4];  // scene node ids
    float t, w[4], n[3];
};

inline bool impactBefore(const Impact& a, const Impact& b) {
    if (a.t != b.t) return a.t < b.t;
    for (int i = 0; i < 4; i++)
        if (a.nodes[i] != b.nodes[i]) return a.nodes[i] < b.nodes[i];
    return a.type < b.type;
}

// newtonsMethod (CollisionHelper.cu:3-20)
inline float newtonsMethod(float a, float b, float c, float d, float x0, int dir) {
    if (dir != 0) {
        float y0 = d + x0 * (c + x0 * (b + x0 * a));
        float ddy0 = 2.0f * b + x0 * (6.0f * a);
        x0 += (float)dir * std::sqrt(ab(2.0f * y0 / ddy0));
    }
    for (int iter = 0; iter < 100; iter++) {
        float y = d + x0 * (c + x0 * (b + x0 * a));
        float dy = c + x0 * (2.0f * b + 3.0f * x0 * a);
        if (dy == 0) return x0;
        float x1 = x0 - y / dy;
        if (ab(x0 - x1) < 1e-6f) return x0;
        x0 = x1;
    }
    return x0;
}

// solveQuadratic (CollisionHelper.cu:22-37)
inline int solveQuadratic(float a, float b, float c, float x[2]) {
    float d = b * b - 4.0f * a * c;
    if (d < 0.0f) {
        x[0] = -b / (2.0f * a);
        return 0;
    }
    float q = -(b + (float)(b < 0.0f ? -1 : 1) * std::sqrt(d)) * 0.5f;
    int i = 0;
    if (ab(a) > 1e-12f * ab(q)) x[i++] = q / a;
    if (ab(q) > 1e-12f * ab(c)) x[i++] = c / q;
    if (i == 2 && x[0] > x[1]) std::swap(x[0], x[1]);
    return i;
}

// solveCubic (CollisionHelper.cu:39-59).  solveQuadratic returns no root without writing one
// when both of its root guards fail (a degenerate derivative: a, b, c all ~0); the reference
// then starts Newton's method from an uninitialised value.  Here that start is 0 (the cubic is
// then constant: Newton stops at once and t = 0 is tested).
inline int solveCubic(float a, float b, float c, float d, float x[3]) {
    float xc[2] = {0.0f, 0.0f};
    int n = solveQuadratic(3.0f * a, 2.0f * b, c, xc);
    if (n == 0) {
        x[0] = newtonsMethod(a, b, c, d, xc[0], 0);
        return 1;
    } else if (n == 1) {
        return solveQuadratic(b, c, d, x);
    } else {
        float yc[2] = {d + xc[0] * (c + xc[0] * (b + xc[0] * a)), d + xc[1] * (c + xc[1] * (b + xc[1] * a))};
        int i = 0;
        if (yc[0] * a >= 0.0f) x[i++] = newtonsMethod(a, b, c, d, xc[0], -1);
        if (yc[0] * yc[1] <= 0.0f) {
            int closer = ab(yc[0]) < ab(yc[1]) ? 0 : 1;
            x[i++] = newtonsMethod(a, b, c, d, xc[closer], closer == 0 ? 1 : -1);
        }
        if (yc[1] * a <= 0.0f) x[i++] = newtonsMethod(a, b, c, d, xc[1], 1);
        return i;
    }
}

template <class T>
inline T mixed3(const V3<T>& a, const V3<T>& b, const V3<T>& c) { return dot(a, cross(b, c)); }  // MathHelper.cuh:43-45

// checkImpact (CollisionHelper.cu:61-110): p = start positions, q = end positions of the four nodes.
inline bool checkImpact(int type, const V3<float> p[4], const V3<float> q[4], Impact& imp) {
    const V3<float> x0 = p[0];
    const V3<float> v0 = sub(q[0], x0);
    const V3<float> x1 = sub(p[1], x0), x2 = sub(p[2], x0), x3 = sub(p[3], x0);
    // relative velocities (the reference's v1, v2, v3)
    const V3<float> u1 = sub(sub(q[1], p[1]), v0), u2 = sub(sub(q[2], p[2]), v0), u3 = sub(sub(q[3], p[3]), v0);
    const float a0 = mixed3(x1, x2, x3);
    const float a1 = mixed3(u1, x2, x3) + mixed3(x1, u2, x3) + mixed3(x1, x2, u3);
    const float a2 = mixed3(x1, u2, u3) + mixed3(u1, x2, u3) + mixed3(u1, u2, x3);
    const float a3 = mixed3(u1, u2, u3);
    float t[3] = {0.0f, 0.0f, 0.0f};
    const int ns = solveCubic(a3, a2, a1, a0, t);
    imp.type = type;
    for (int i = 0; i < ns; i++) {
        if (t[i] < 0.0f || t[i] > 1.0f) continue;
        V3<float> y[4];
        for (int k = 0; k < 4; k++) y[k] = add(p[k], scl(t[i], sub(q[k], p[k])));  // Node::position
        V3<float> n;
        float w[4], h;
        bool ok, inside;
        if (type == 0) {
            ok = signedVertexFace(y[0], y[1], y[2], y[3], n, w, h);
            inside = ok && (mn(-w[1], mn(-w[2], -w[3])) >= -1e-6f);
        } else {
            ok = signedEdgeEdge(y[0], y[1], y[2], y[3], n, w, h);
            inside = ok && (mn(mn(w[0], w[1]), mn(-w[2], -w[3])) >= -1e-6f);
        }
        if (!ok) continue;  // INFINITY distance: never an impact
        if (dot(n, add(add(scl(w[1], u1), scl(w[2], u2)), scl(w[3], u3))) > 0.0f) n = v3(-n[0], -n[1], -n[2]);
        if (ab(h) < 1e-6f && inside) {
            imp.t = t[i];
            for (int k = 0; k < 4; k++) imp.w[k] = w[k];
            for (int k = 0; k < 3; k++) imp.n[k] = n[k];
            return true;
        }
    }
    return false;
}

// Scene state for the collision step: the detection view (x = current positions) plus x0 and
// lumped masses.
struct CollideScene {
    DetectScene S;
    std::vector<float> x0, mass;
    V3<float> X0(int i) const { return v3(x0[3 * i], x0[3 * i + 1], x0[3 * i + 2]); }
};

class Collider {
public:
    // Optional replacements (the reference adapter's): the impact check with its bounds test
    // (type, a, b -> impact: vertex-face a = node, b = face; edge-edge a, b = edges), and the
    // projection of one round (impacts, thickness, positions in/out).
    std::function<bool(int, int, int, float, Impact&)> impactHook;
    std::function<void(const std::vector<Impact>&, float, std::vector<float>&)> optimizeHook;

    explicit Collider(CollideScene& c) : C(c) {}

    CollideScene& C;

    // Bounds of the x0 and x positions (ccd bounds) of a node set.
    void boxOf(const int* nodes, int k, float lo[3], float hi[3]) const {
        for (int c = 0; c < 3; c++) {
            lo[c] = 3.0e38f;
            hi[c] = -3.0e38f;
        }
        for (int i = 0; i < k; i++)
            for (int c = 0; c < 3; c++) {
                const float a = C.S.x[3 * nodes[i] + c], b = C.x0[3 * nodes[i] + c];
                lo[c] = mn(mn(lo[c], a), b);
                hi[c] = mx(mx(hi[c], a), b);
            }
    }
    static bool overlap(const float alo[3], const float ahi[3], const float blo[3], const float bhi[3], float t) {
        for (int c = 0; c < 3; c++) {  // Bounds::overlap(b, thickness): a against b dilated
            if (alo[c] > bhi[c] + t) return false;
            if (ahi[c] < blo[c] - t) return false;
        }
        return true;
    }

    // checkVertexFaceImpact / checkEdgeEdgeImpact (CollisionHelper.cu:112-136)
    bool impact(int type, int a, int b, float thickness, Impact& imp) const {
        if (impactHook) return impactHook(type, a, b, thickness, imp);
        int nodes[4];
        float alo[3], ahi[3], blo[3], bhi[3];
        if (type == 0) {
            const int* y = &C.S.fx[3 * b];
            if (a == y[0] || a == y[1] || a == y[2]) return false;
            nodes[0] = a;
            nodes[1] = y[0];
            nodes[2] = y[1];
            nodes[3] = y[2];
            boxOf(nodes, 1, alo, ahi);
            boxOf(nodes + 1, 3, blo, bhi);
        } else {
            nodes[0] = C.S.eNodes[2 * a];
            nodes[1] = C.S.eNodes[2 * a + 1];
            nodes[2] = C.S.eNodes[2 * b];
            nodes[3] = C.S.eNodes[2 * b + 1];
            if (nodes[0] == nodes[2] || nodes[0] == nodes[3] || nodes[1] == nodes[2] || nodes[1] == nodes[3]) return false;
            boxOf(nodes, 2, alo, ahi);
            boxOf(nodes + 2, 2, blo, bhi);
        }
        if (!overlap(alo, ahi, blo, bhi, thickness)) return false;
        V3<float> p[4], q[4];
        for (int k = 0; k < 4; k++) {
            p[k] = C.X0(nodes[k]);
            q[k] = C.S.X(nodes[k]);
        }
        if (!checkImpact(type, p, q, imp)) return false;
        for (int k = 0; k < 4; k++) imp.nodes[k] = nodes[k];
        return true;
    }

    // findImpacts (Simulator.cu:369-392): every candidate face pair's 6 vertex-face and 9
    // edge-edge checks.
    std::vector<Impact> findImpacts(float thickness) const {
        const int nf = C.S.nFaces();
        std::vector<float> lo(3 * (size_t)nf), hi(3 * (size_t)nf);
        for (int f = 0; f < nf; f++) boxOf(&C.S.fx[3 * f], 3, &lo[3 * f], &hi[3 * f]);
        std::vector<int> order(nf);
        for (int f = 0; f < nf; f++) order[f] = f;
        std::sort(order.begin(), order.end(), [&](int a, int b) { return lo[3 * a] < lo[3 * b]; });
        std::vector<Impact> out;
        Impact imp{};
        for (int i = 0; i < nf; i++) {
            const int a = order[i];
            for (int j = i + 1; j < nf; j++) {
                const int b = order[j];
                if (lo[3 * b] > hi[3 * a] + 2.0f * thickness) break;
                if (C.S.faceGroup[a] != C.S.faceGroup[b]) continue;
                const int f0 = std::min(a, b), f1 = std::max(a, b);
                if (!overlap(&lo[3 * f1], &hi[3 * f1], &lo[3 * f0], &hi[3 * f0], thickness)) continue;
                for (int k = 0; k < 3; k++)
                    if (impact(0, C.S.fx[3 * f0 + k], f1, thickness, imp)) out.push_back(imp);
                for (int k = 0; k < 3; k++)
                    if (impact(0, C.S.fx[3 * f1 + k], f0, thickness, imp)) out.push_back(imp);
                for (int k = 0; k < 3; k++)
                    for (int l = 0; l < 3; l++)
                        if (impact(1, C.S.fEdges[3 * f0 + k], C.S.fEdges[3 * f1 + l], thickness, imp)) out.push_back(imp);
            }
        }
        return out;
    }

    // independentImpacts (Simulator.cu:394-420): by impact time, each node in one impact at most.
    static std::vector<Impact> independent(std::vector<Impact> imps, int nNodes) {
        std::sort(imps.begin(), imps.end(), impactBefore);
        std::vector<char> used(nNodes, 0);
        std::vector<Impact> out;
        for (const Impact& m : imps) {
            bool ok = true;
            for (int k = 0; k < 4; k++) ok &= !used[m.nodes[k]];
            if (!ok) continue;
            out.push_back(m);
            for (int k = 0; k < 4; k++) used[m.nodes[k]] = 1;
        }
        return out;
    }

    // CollisionOptimization (CollisionOptimization.cu:5-36, 61-131) solved by
    // Optimization::solve (Optimization.cu:24-137); x1 = positions when the step began.
    void optimize(const std::vector<Impact>& imps, float thickness, const std::vector<float>& x1) {
        if (optimizeHook) {
            optimizeHook(imps, thickness, C.S.x);
            return;
        }
        const int nc = (int)imps.size();
        std::vector<int> nodes;
        for (const Impact& m : imps)
            for (int k = 0; k < 4; k++) nodes.push_back(m.nodes[k]);
        std::sort(nodes.begin(), nodes.end());
        nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
        const int nn = (int)nodes.size();
        std::vector<int> idx(4 * (size_t)nc);
        for (int c = 0; c < nc; c++)
            for (int k = 0; k < 4; k++)
                idx[4 * c + k] = (int)(std::lower_bound(nodes.begin(), nodes.end(), imps[c].nodes[k]) - nodes.begin());
        float invMass = 0.0f;
        for (int i = 0; i < nn; i++) invMass += 1.0f / C.mass[nodes[i]];
        invMass /= (float)nn;
        auto P1 = [&](int i) { return v3(x1[3 * nodes[i]], x1[3 * nodes[i] + 1], x1[3 * nodes[i] + 2]); };
        auto nrm = [&](int c) { return v3(imps[c].n[0], imps[c].n[1], imps[c].n[2]); };
        const float mu = 1e3f;
        std::vector<float> lambda(nc, 0.0f);
        auto constraint = [&](const std::vector<V3<float>>& x, int c) {
            float a = -thickness;
            for (int k = 0; k < 4; k++) a += imps[c].w[k] * dot(nrm(c), x[idx[4 * c + k]]);
            return a;
        };
        auto clampV = [](float v) { return mn(v, 0.0f); };  // clampViolation(x, +1)
        auto objective = [&](const std::vector<V3<float>>& x) {
            float a = 0.0f;
            for (int i = 0; i < nn; i++) a += C.mass[nodes[i]] * norm2(sub(x[i], P1(i)));
            return 0.5f * a * invMass;
        };
        auto value = [&](const std::vector<V3<float>>& x) {
            float a = objective(x);
            for (int c = 0; c < nc; c++) {
                const float coef = clampV(constraint(x, c) + lambda[c] / mu);
                if (coef != 0.0f) a += 0.5f * mu * (coef * coef);
            }
            return a;
        };
        std::vector<V3<float>> cur(nn), next(nn), grad(nn);
        for (int i = 0; i < nn; i++) cur[i] = C.S.X(nodes[i]);
        float f, ft = 0.0f, s = 1e-3f * (float)nn;
        for (int iter = 0; iter < kMaxOptIterations; iter++) {
            f = objective(cur);
            for (int i = 0; i < nn; i++) grad[i] = scl(invMass * C.mass[nodes[i]], sub(cur[i], P1(i)));
            for (int c = 0; c < nc; c++) {
                const float coef = clampV(constraint(cur, c) + lambda[c] / mu);
                if (coef != 0.0f) {
                    f += 0.5f * mu * (coef * coef);
                    const float factor = mu * coef;
                    for (int k = 0; k < 4; k++) grad[idx[4 * c + k]] = add(grad[idx[4 * c + k]], scl(factor * imps[c].w[k], nrm(c)));
                }
            }
            float g2 = 0.0f;
            for (int i = 0; i < nn; i++) g2 += norm2(grad[i]);
            s /= 0.7f;
            do {
                s *= 0.7f;
                for (int i = 0; i < nn; i++) next[i] = sub(cur[i], scl(s, grad[i]));
                ft = value(next);
            } while (ft >= f - 0.5f * s * g2 && s >= kEpsS && ab(f - ft) >= kEpsF);
            if (s < kEpsS || ab(f - ft) < kEpsF) break;
            cur = next;
            for (int c = 0; c < nc; c++) lambda[c] = clampV(lambda[c] + mu * constraint(cur, c));
        }
        for (int i = 0; i < nn; i++)
            for (int c = 0; c < 3; c++) C.S.x[3 * nodes[i] + c] = cur[i][c];
    }

    // Simulator::collisionStep (Simulator.cu:640-684); returns the rounds run, or -1 when the
    // impacts were not resolved.  impactsTotal receives the impacts accumulated.
    int run(float thickness, float dt, int& impactsTotal, int maxRounds = kMaxCollisionRounds) {
        const std::vector<float> x1 = C.S.x;
        int rounds = 0;
        bool success = false;
        impactsTotal = 0;
        for (int deform = 0; deform < 2 && !success; deform++) {
            std::vector<Impact> imps;
            for (int i = 0; i < kMaxCollisionRounds && rounds < 2 * maxRounds; i++) {
                if (i >= maxRounds) break;
                rounds++;
                std::vector<Impact> fresh = findImpacts(thickness);
                if (fresh.empty()) {
                    success = true;
                    break;
                }
                fresh = independent(fresh, C.S.nNodes());
                imps.insert(imps.end(), fresh.begin(), fresh.end());
                impactsTotal += (int)fresh.size();
                optimize(imps, thickness, x1);
            }
        }
        return success ? rounds : -1;
    }
};

}  // namespace orc

#endif
