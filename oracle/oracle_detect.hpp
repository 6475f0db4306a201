// Proximity detection restated for the CPU oracle.  TEST INFRASTRUCTURE ONLY: nothing in
// the product library includes this file.
//
// Restates what Simulator::physicsStep runs before the cloth steps (Simulator.cu:571-586):
// findProximities (Simulator.cu:271-298, with the output order of findProximitiesGpu,
// :300-349: node proximities by (node, side), then edge proximities by (edge, side), then
// face proximities by (face, side), index order standing for the reference's pointer order)
// over the face pairs its BVH traversal reports (Simulator.cu:168-177, BVHNode.cu:40-63:
// every pair of faces of one cloth, or of two cloths, whose bounds overlap after dilating
// one of them by 2 x repulsionThickness; which pairs these are does not depend on the tree,
// so the oracle finds them by a sweep over sorted bounds), the tests checkVertexFaceProximity
// and checkEdgeEdgeProximity (Simulator.cu:198-261), signedVertexFaceDistance and
// signedEdgeEdgeDistance (MathHelper.cu:38-69), inEdge (PhysicsHelper.cu:3-18), and the
// Proximity constructors (Proximity.cu:5-21).  Node normals and areas follow
// Mesh::updateNodeGeometries (Mesh.cu:182-203), face normals Face::update (Face.cu:124-132),
// edge areas Edge::area (Edge.cu:89-95).  Cloth nodes are free (Mesh.cu:349), so every
// proximity gets the cloth friction.  Min-reductions keep (distance, other element) pairs
// and break distance ties by the other element's index.
//
// Hooks let the reference adapter substitute the reference's own predicates.
#ifndef CLOTHSTEP_ORACLE_DETECT_HPP
#define CLOTHSTEP_ORACLE_DETECT_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <utility>
#include <vector>

#include "oracle_math.hpp"
#include "oracle_system.hpp"

namespace orc {

// signedVertexFaceDistance (MathHelper.cu:38-52); returns false where the reference returns
// INFINITY (degenerate face: the test then never yields a proximity).
template <class T>
inline bool signedVertexFace(const V3<T>& x, const V3<T>& y0, const V3<T>& y1, const V3<T>& y2, V3<T>& n, T w[4],
                             T& h) {
    n = cross(normalized(sub(y1, y0)), normalized(sub(y2, y0)));
    if (norm2(n) < T(1e-6f)) return false;
    n = normalized(n);
    h = dot(sub(x, y0), n);
    const T b0 = dot(sub(y1, x), cross(sub(y2, x), n));
    const T b1 = dot(sub(y2, x), cross(sub(y0, x), n));
    const T b2 = dot(sub(y0, x), cross(sub(y1, x), n));
    w[0] = T(1);
    w[1] = -b0 / (b0 + b1 + b2);
    w[2] = -b1 / (b0 + b1 + b2);
    w[3] = -b2 / (b0 + b1 + b2);
    return true;
}

// signedEdgeEdgeDistance (MathHelper.cu:54-69).
template <class T>
inline bool signedEdgeEdge(const V3<T>& x0, const V3<T>& x1, const V3<T>& y0, const V3<T>& y1, V3<T>& n, T w[4],
                           T& h) {
    n = cross(normalized(sub(x1, x0)), normalized(sub(y1, y0)));
    if (norm2(n) < T(1e-6f)) return false;
    n = normalized(n);
    h = dot(sub(x0, y0), n);
    const T a0 = dot(sub(y1, x1), cross(sub(y0, x1), n));
    const T a1 = dot(sub(y0, x0), cross(sub(y1, x0), n));
    const T b0 = dot(sub(x0, y1), cross(sub(x1, y1), n));
    const T b1 = dot(sub(x1, y0), cross(sub(x0, y0), n));
    w[0] = a0 / (a0 + a1);
    w[1] = a1 / (a0 + a1);
    w[2] = -b0 / (b0 + b1);
    w[3] = -b1 / (b0 + b1);
    return true;
}

// One detected proximity, in the form Cloth::physicsStep receives it (Proximity.cuh:11-21).
struct DetectedProximity {
    int nodes[4];  // scene node ids (cloths concatenated)
    float n[3], w[4], mu, stiffness;
    float depth;   // the reduced distance that admitted it
    int kind;      // 0 node key, 1 edge key, 2 face key
};

struct DetectParams {
    float repulsionThickness = 1e-3f;   // Magic.cu:8
    float collisionStiffness = 1e9f;    // Magic.cu:7
    float clothFriction = 0.6f;         // Simulator.cu:25
};

// Scene-wide view of the cloths: nodes, faces and edges renumbered consecutively in cloth order.
struct DetectScene {
    std::vector<float> x;                  // 3 per node
    std::vector<int> fx;                   // 3 per face (scene node ids)
    std::vector<int> fEdges;               // 3 per face: edges (v0 v1), (v1 v2), (v2 v0)
    std::vector<int> eNodes, eFace;        // 2 per edge; eFace -1 where no face
    std::vector<float> farea;              // rest area per face (Face.cu:17)
    std::vector<int> faceGroup;            // collision group of each face's cloth
    // derived (prepare)
    std::vector<float> fn, nn, narea, earea;

    void addCloth(const Topology& t, const float* xs, const float* fareas, int group) {
        const int n0 = (int)(x.size() / 3), f0 = (int)(fx.size() / 3), e0 = (int)(eNodes.size() / 2);
        x.insert(x.end(), xs, xs + 3 * t.nNodes);
        std::map<std::pair<int, int>, int> emap;
        for (int e = 0; e < t.nEdges(); e++) {
            emap[{t.eNodes[2 * e], t.eNodes[2 * e + 1]}] = e;
            eNodes.push_back(n0 + t.eNodes[2 * e]);
            eNodes.push_back(n0 + t.eNodes[2 * e + 1]);
            for (int s = 0; s < 2; s++) eFace.push_back(t.eFace[2 * e + s] < 0 ? -1 : f0 + t.eFace[2 * e + s]);
        }
        auto eid = [&](int a, int b) { return emap.at({std::min(a, b), std::max(a, b)}); };
        for (int f = 0; f < t.nFaces; f++) {
            const int* v = &t.fx[3 * f];
            for (int k = 0; k < 3; k++) fx.push_back(n0 + v[k]);
            fEdges.push_back(e0 + eid(v[0], v[1]));
            fEdges.push_back(e0 + eid(v[1], v[2]));
            fEdges.push_back(e0 + eid(v[2], v[0]));
            farea.push_back(fareas[f]);
            faceGroup.push_back(group);
        }
    }

    V3<float> X(int i) const { return v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]); }
    V3<float> FN(int f) const { return v3(fn[3 * f], fn[3 * f + 1], fn[3 * f + 2]); }
    V3<float> NN(int i) const { return v3(nn[3 * i], nn[3 * i + 1], nn[3 * i + 2]); }
    int nNodes() const { return (int)(x.size() / 3); }
    int nFaces() const { return (int)(fx.size() / 3); }
    int nEdges() const { return (int)(eNodes.size() / 2); }

    // Face::update normals, Mesh::updateNodeGeometries normals and areas (faces in index
    // order), Edge::area.
    void prepare() {
        const int nf = nFaces(), nn_ = nNodes(), ne = nEdges();
        fn.assign(3 * nf, 0.0f);
        for (int f = 0; f < nf; f++) {
            V3<float> n = faceNormal(X(fx[3 * f]), X(fx[3 * f + 1]), X(fx[3 * f + 2]));
            for (int c = 0; c < 3; c++) fn[3 * f + c] = n[c];
        }
        std::vector<V3<float>> acc(nn_, v3(0.0f, 0.0f, 0.0f));
        narea.assign(nn_, 0.0f);
        for (int f = 0; f < nf; f++) {
            const float a = farea[f] / 3.0f;
            for (int i = 0; i < 3; i++) {
                const int node = fx[3 * f + i];
                const V3<float> e0 = sub(X(fx[3 * f + (i + 1) % 3]), X(node));
                const V3<float> e1 = sub(X(fx[3 * f + (i + 2) % 3]), X(node));
                acc[node] = add(acc[node], dvd(cross(e0, e1), norm2(e0) * norm2(e1)));
                narea[node] += a;
            }
        }
        nn.assign(3 * nn_, 0.0f);
        for (int i = 0; i < nn_; i++) {
            V3<float> n = normalized(acc[i]);
            for (int c = 0; c < 3; c++) nn[3 * i + c] = n[c];
        }
        earea.assign(ne, 0.0f);
        for (int e = 0; e < ne; e++) {
            float a = 0.0f;
            for (int s = 0; s < 2; s++)
                if (eFace[2 * e + s] >= 0) a += farea[eFace[2 * e + s]];
            earea[e] = a;
        }
    }
};

class Detector {
public:
    // Optional replacements of the predicates (the reference adapter's): vertex-face distance
    // (node, face), edge-edge distance (edge0, edge1), inEdge(w, edge0, edge1), and the
    // Proximity constructors (node, face) and (edge0, edge1).
    std::function<bool(int, int, V3<float>&, float*, float&)> vfHook;
    std::function<bool(int, int, V3<float>&, float*, float&)> eeHook;
    std::function<bool(float, int, int)> inEdgeHook;
    std::function<void(int, int, const DetectParams&, DetectedProximity&)> proxVFHook, proxEEHook;

    explicit Detector(const DetectScene& s) : S(s) {}

    std::vector<DetectedProximity> run(const DetectParams& P) {
        const float thick = 2.0f * P.repulsionThickness;  // Simulator.cu:274
        nodeKey.assign(2 * (size_t)S.nNodes(), kNone);
        edgeKey.assign(2 * (size_t)S.nEdges(), kNone);
        faceKey.assign(2 * (size_t)S.nFaces(), kNone);
        forEachPair(thick, [&](int f0, int f1) { checkFaces(f0, f1); });
        std::vector<DetectedProximity> out;
        auto admit = [&](uint64_t v) { return v != kNone && dist(v) < 2.0f * P.repulsionThickness; };
        for (size_t k = 0; k < nodeKey.size(); k++)
            if (admit(nodeKey[k])) out.push_back(makeVF((int)(k / 2), other(nodeKey[k]), P, 0, dist(nodeKey[k])));
        for (size_t k = 0; k < edgeKey.size(); k++)
            if (admit(edgeKey[k])) out.push_back(makeEE((int)(k / 2), other(edgeKey[k]), P, dist(edgeKey[k])));
        for (size_t k = 0; k < faceKey.size(); k++)
            if (admit(faceKey[k])) out.push_back(makeVF(other(faceKey[k]), (int)(k / 2), P, 2, dist(faceKey[k])));
        return out;
    }

    // Candidate face pairs (each unordered pair once, lower index first) whose bounds overlap
    // after dilating the first by `thick` (Bounds.cu:85-101), within a collision group.
    void forEachPair(float thick, const std::function<void(int, int)>& fn) const {
        const int nf = S.nFaces();
        std::vector<float> lo(3 * (size_t)nf), hi(3 * (size_t)nf);
        for (int f = 0; f < nf; f++)
            for (int c = 0; c < 3; c++) {
                float a = S.x[3 * S.fx[3 * f] + c], b = S.x[3 * S.fx[3 * f + 1] + c], d = S.x[3 * S.fx[3 * f + 2] + c];
                lo[3 * f + c] = mn(mn(a, b), d);
                hi[3 * f + c] = mx(mx(a, b), d);
            }
        std::vector<int> order(nf);
        for (int f = 0; f < nf; f++) order[f] = f;
        std::sort(order.begin(), order.end(), [&](int a, int b) { return lo[3 * a] < lo[3 * b]; });
        auto overlap = [&](int a, int b) {  // a's bounds against b's dilated by thick
            for (int c = 0; c < 3; c++) {
                if (lo[3 * a + c] > hi[3 * b + c] + thick) return false;
                if (hi[3 * a + c] < lo[3 * b + c] - thick) return false;
            }
            return true;
        };
        for (int i = 0; i < nf; i++) {
            const int a = order[i];
            for (int j = i + 1; j < nf; j++) {
                const int b = order[j];
                // sorted by lower x: no later face can pass the x test (margin for rounding)
                if (lo[3 * b] > hi[3 * a] + 2.0f * thick) break;
                if (S.faceGroup[a] != S.faceGroup[b]) continue;
                const int f0 = std::min(a, b), f1 = std::max(a, b);
                if (overlap(f1, f0)) fn(f0, f1);
            }
        }
    }

private:
    static constexpr uint64_t kNone = ~0ULL;
    const DetectScene& S;
    std::vector<uint64_t> nodeKey, edgeKey, faceKey;

    static uint64_t pack(float d, int other) {
        if (d == 0.0f) d = 0.0f;  // -0 compares equal to +0
        uint32_t bits;
        std::memcpy(&bits, &d, 4);
        return (uint64_t)bits << 32 | (uint32_t)other;
    }
    static float dist(uint64_t v) {
        uint32_t bits = (uint32_t)(v >> 32);
        float d;
        std::memcpy(&d, &bits, 4);
        return d;
    }
    static int other(uint64_t v) { return (int)(uint32_t)v; }
    static void keep(uint64_t& slot, uint64_t v) { slot = std::min(slot, v); }

    bool vf(int node, int face, V3<float>& n, float w[4], float& h) const {
        if (vfHook) return vfHook(node, face, n, w, h);
        return signedVertexFace(S.X(node), S.X(S.fx[3 * face]), S.X(S.fx[3 * face + 1]), S.X(S.fx[3 * face + 2]), n, w, h);
    }
    bool ee(int e0, int e1, V3<float>& n, float w[4], float& h) const {
        if (eeHook) return eeHook(e0, e1, n, w, h);
        return signedEdgeEdge(S.X(S.eNodes[2 * e0]), S.X(S.eNodes[2 * e0 + 1]), S.X(S.eNodes[2 * e1]),
                              S.X(S.eNodes[2 * e1 + 1]), n, w, h);
    }
    // inEdge (PhysicsHelper.cu:3-18)
    bool inEdge(float w, int e0, int e1) const {
        if (inEdgeHook) return inEdgeHook(w, e0, e1);
        const V3<float> x = add(scl(1.0f - w, S.X(S.eNodes[2 * e0])), scl(w, S.X(S.eNodes[2 * e0 + 1])));
        bool in = true;
        for (int i = 0; i < 2; i++) {
            const int face = S.eFace[2 * e1 + i];
            if (face < 0) continue;
            const int node0 = S.eNodes[2 * e1 + i], node1 = S.eNodes[2 * e1 + 1 - i];
            const V3<float> e = sub(S.X(node1), S.X(node0));
            const V3<float> r = sub(x, S.X(node0));
            in &= (dot(e, cross(S.FN(face), r)) >= 0.0f);
        }
        return in;
    }

    // checkVertexFaceProximity (Simulator.cu:198-229)
    void checkVF(int node, int face) {
        const int* y = &S.fx[3 * face];
        if (node == y[0] || node == y[1] || node == y[2]) return;
        V3<float> n;
        float w[4], h;
        if (!vf(node, face, n, w, h)) return;
        const float d = ab(h);
        const bool inside = (mn(-w[1], mn(-w[2], -w[3])) >= 1e-6f);
        if (!inside) return;
        const int sideN = dot(n, S.NN(node)) >= 0.0f ? 0 : 1;
        keep(nodeKey[2 * (size_t)node + sideN], pack(d, face));
        const int sideF = -dot(n, S.FN(face)) >= 0.0f ? 0 : 1;
        keep(faceKey[2 * (size_t)face + sideF], pack(d, node));
    }

    // checkEdgeEdgeProximity (Simulator.cu:231-261)
    void checkEE(int e0, int e1) {
        const int a0 = S.eNodes[2 * e0], a1 = S.eNodes[2 * e0 + 1], b0 = S.eNodes[2 * e1], b1 = S.eNodes[2 * e1 + 1];
        if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) return;
        V3<float> n;
        float w[4], h;
        if (!ee(e0, e1, n, w, h)) return;
        const float d = ab(h);
        const bool inside = (mn(mn(w[0], w[1]), mn(-w[2], -w[3])) >= 1e-6f && inEdge(w[1], e0, e1) && inEdge(-w[3], e1, e0));
        if (!inside) return;
        const int side0 = dot(n, add(S.NN(a0), S.NN(a1))) >= 0.0f ? 0 : 1;
        keep(edgeKey[2 * (size_t)e0 + side0], pack(d, e1));
        const int side1 = -dot(n, add(S.NN(b0), S.NN(b1))) >= 0.0f ? 0 : 1;
        keep(edgeKey[2 * (size_t)e1 + side1], pack(d, e0));
    }

    // checkProximities (Simulator.cu:263-269)
    void checkFaces(int f0, int f1) {
        for (int i = 0; i < 3; i++) checkVF(S.fx[3 * f0 + i], f1);
        for (int i = 0; i < 3; i++) checkVF(S.fx[3 * f1 + i], f0);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) checkEE(S.fEdges[3 * f0 + i], S.fEdges[3 * f1 + j]);
    }

    // Proximity(node, face) (Proximity.cu:5-12)
    DetectedProximity makeVF(int node, int face, const DetectParams& P, int kind, float depth) const {
        DetectedProximity r{};
        r.kind = kind;
        r.depth = depth;
        if (proxVFHook) {
            proxVFHook(node, face, P, r);
        } else {
            r.nodes[0] = node;
            for (int k = 0; k < 3; k++) r.nodes[1 + k] = S.fx[3 * face + k];
            r.stiffness = P.collisionStiffness * mn(S.narea[node], S.farea[face]);
            V3<float> n;
            float h;
            signedVertexFace(S.X(node), S.X(S.fx[3 * face]), S.X(S.fx[3 * face + 1]), S.X(S.fx[3 * face + 2]), n, r.w, h);
            if (h < 0.0f) n = v3(-n[0], -n[1], -n[2]);
            for (int c = 0; c < 3; c++) r.n[c] = n[c];
            r.mu = P.clothFriction;
        }
        return r;
    }

    // Proximity(edge0, edge1) (Proximity.cu:14-21)
    DetectedProximity makeEE(int e0, int e1, const DetectParams& P, float depth) const {
        DetectedProximity r{};
        r.kind = 1;
        r.depth = depth;
        if (proxEEHook) {
            proxEEHook(e0, e1, P, r);
        } else {
            r.nodes[0] = S.eNodes[2 * e0];
            r.nodes[1] = S.eNodes[2 * e0 + 1];
            r.nodes[2] = S.eNodes[2 * e1];
            r.nodes[3] = S.eNodes[2 * e1 + 1];
            r.stiffness = P.collisionStiffness * mn(S.earea[e0], S.earea[e1]);
            V3<float> n;
            float h;
            signedEdgeEdge(S.X(r.nodes[0]), S.X(r.nodes[1]), S.X(r.nodes[2]), S.X(r.nodes[3]), n, r.w, h);
            if (h < 0.0f) n = v3(-n[0], -n[1], -n[2]);
            for (int c = 0; c < 3; c++) r.n[c] = n[c];
            r.mu = P.clothFriction;
        }
        return r;
    }
};

}  // namespace orc

#endif
