// Reference adapter (oracle/_ref/libclothref.so).  TEST INFRASTRUCTURE ONLY.
//
// Compiled together with the reference's own sources, read in place from the reference
// checkout (Node.cu, Vertex.cu, Face.cu, Edge.cu, Material.cu, MathHelper.cu,
// JsonHelper.cu, PhysicsHelper.cu, ...; see oracle/Makefile).  It builds the reference's
// Node/Vertex/Face/Edge objects the way Mesh::load does on the CPU (Mesh.cu:360-399) and
// evaluates forces and Jacobians with the reference's stretchingForce
// (PhysicsHelper.cu:264-291) and bendingForce (PhysicsHelper.cu:327-353), face rest data
// with Face::initialize (Face.cu:12-20), normals with Face::update (Face.cu:124-132) and
// stiffness with Material (Material.cu:3-156).  Assembly and the FP32 sparse Cholesky
// around them are the oracle's restatement of Cloth.cu:42-169 and of SimplicialLLT.
// The exported names mirror liboracle.so's with the prefix ref_.
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <sstream>
#include <thread>
#include <unordered_map>
#include <vector>

#include "CollisionHelper.cuh"
#include "CollisionOptimization.cuh"
#include "Edge.cuh"
#include "Face.cuh"
#include "Material.cuh"
#include "Motion.cuh"
#include "Node.cuh"
#include "PhysicsHelper.cuh"
#include "Proximity.cuh"
#include "Transformation.cuh"
#include "Vertex.cuh"

#include "oracle_collide.hpp"
#include "oracle_detect.hpp"
#include "oracle_system.hpp"

// The reference's global CPU/GPU switch (main.cu:7): the CPU branches of the optimization run.
bool gpu = false;

namespace {
struct ClothBase;
}
// Install the reference's own detection predicates and collision step parts (defined below).
static void orcDetectHooks(orc::Detector& D, const std::vector<ClothBase*>& cloths, const orc::DetectScene& S);
static void orcCollideHooks(orc::Collider& K, const std::vector<ClothBase*>& cloths, orc::CollideScene& S);
#define ORC_DETECT_HOOKS 1
#define ORC_COLLIDE_HOOKS 1
#define ORC_API(name) ref_##name
#define ORC_NO_DEFAULT_FACTORIES 1
#include "oracle_capi.inc"

namespace {

struct RefCloth {
    std::vector<Node> nodes;
    std::vector<Vertex> verts;
    std::vector<Face> faces;
    std::vector<Edge> edges;
    const ::Material* mat = nullptr;
};

struct RefClothImpl : ClothImpl<float> {
    RefCloth rc;
};

}  // namespace

extern "C" {

// Transformation(json).applyToPoint (Transformation.cu:8-13, 82-84) of n points; json_text: a
// "transform" object ({"scale", "translate", "rotate": [degrees, axis]}).
void ref_transform_points(const char* json_text, int n, const double* p, double* out) {
    Json::Value v;
    std::istringstream in(json_text);
    in >> v;
    const Transformation t(v);
    for (int i = 0; i < n; i++) {
        const Vector3f q = t.applyToPoint(Vector3f((float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2]));
        for (int c = 0; c < 3; c++) out[3 * i + c] = q(c);
    }
}

// Motion(json).computeTransformation(time) (Motion.cu:3-72) applied to n points, for each of
// n_times increasing times on one Motion (its segment index advances as the reference's does);
// json_text: a "motions" entry (an array of {"time", "transform"} keyframes).
void ref_motion_points(const char* json_text, int n_times, const double* times, int n, const double* p, double* out) {
    Json::Value v;
    std::istringstream in(json_text);
    in >> v;
    Motion m(v);
    for (int k = 0; k < n_times; k++) {
        const Transformation t = m.computeTransformation((float)times[k]);
        for (int i = 0; i < n; i++) {
            const Vector3f q = t.applyToPoint(Vector3f((float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2]));
            for (int c = 0; c < 3; c++) out[3 * (k * n + i) + c] = q(c);
        }
    }
}

// json_text: the cloth's "materials" object, e.g. {"data": "path.json", "thicken": 1}.
void* ref_material_new(const char* json_text) {
    Json::Value v;
    std::istringstream in(json_text);
    in >> v;
    return new ::Material(v);
}

void ref_material_free(void* m) { delete static_cast<::Material*>(m); }

double ref_material_density(void* m) { return static_cast<::Material*>(m)->getDensity(); }

void ref_material_stretching(void* m, int n, const double* G3, double* out) {
    auto* mat = static_cast<::Material*>(m);
    for (int i = 0; i < n; i++) {
        Matrix2x2f G;
        G(0, 0) = (float)G3[3 * i];
        G(0, 1) = G(1, 0) = (float)G3[3 * i + 1];
        G(1, 1) = (float)G3[3 * i + 2];
        Vector4f k = mat->stretchingStiffness(G);
        for (int c = 0; c < 4; c++) out[4 * i + c] = k(c);
    }
}

void ref_material_bending(void* m, int n, const double* in5, double* out) {
    auto* mat = static_cast<::Material*>(m);
    for (int i = 0; i < n; i++) {
        const double* q = in5 + 5 * i;
        out[i] = mat->bendingStiffness((float)q[0], (float)q[1], (float)q[2], Vector2f((float)q[3], (float)q[4]));
    }
}

void* ref_cloth_new(void* mat, int nn, const double* x, const double* v, int nv, const double* u, int nf,
                    const int* fx, const int* fu) {
    auto* c = new RefClothImpl();
    RefCloth& rc = c->rc;
    rc.mat = static_cast<::Material*>(mat);
    rc.nodes.resize(nn);
    for (int i = 0; i < nn; i++) {
        rc.nodes[i] = Node(Vector3f((float)x[3 * i], (float)x[3 * i + 1], (float)x[3 * i + 2]), true);
        rc.nodes[i].v = Vector3f((float)v[3 * i], (float)v[3 * i + 1], (float)v[3 * i + 2]);
        rc.nodes[i].index = i;
    }
    rc.verts.resize(nv);
    for (int i = 0; i < nv; i++) {
        rc.verts[i] = Vertex(Vector2f((float)u[2 * i], (float)u[2 * i + 1]));
        rc.verts[i].index = i;
    }
    // Topology numbering (edge order) comes from the oracle's restatement; the sides are
    // then set by the reference's own Edge::initialize, in Mesh::load's call order.
    orc::Topology topo;
    topo.build(nn, nv, nf, fx, fu);
    std::unordered_map<uint64_t, int> emap;
    for (int e = 0; e < topo.nEdges(); e++)
        emap[(uint64_t)(uint32_t)topo.eNodes[2 * e] << 32 | (uint32_t)topo.eNodes[2 * e + 1]] = e;
    auto eid = [&](int a, int b) {
        if (a > b) std::swap(a, b);
        return emap[(uint64_t)(uint32_t)a << 32 | (uint32_t)b];
    };
    rc.edges.resize(topo.nEdges());
    for (int e = 0; e < topo.nEdges(); e++)
        rc.edges[e] = Edge(&rc.nodes[topo.eNodes[2 * e]], &rc.nodes[topo.eNodes[2 * e + 1]]);
    rc.faces.resize(nf);
    for (int f = 0; f < nf; f++) {
        Vertex* v0 = &rc.verts[fu[3 * f]];
        Vertex* v1 = &rc.verts[fu[3 * f + 1]];
        Vertex* v2 = &rc.verts[fu[3 * f + 2]];
        v0->node = &rc.nodes[fx[3 * f]];
        v1->node = &rc.nodes[fx[3 * f + 1]];
        v2->node = &rc.nodes[fx[3 * f + 2]];
        rc.faces[f] = Face(v0, v1, v2, rc.mat);
        Edge* e0 = &rc.edges[eid(fx[3 * f], fx[3 * f + 1])];
        Edge* e1 = &rc.edges[eid(fx[3 * f + 1], fx[3 * f + 2])];
        Edge* e2 = &rc.edges[eid(fx[3 * f + 2], fx[3 * f])];
        e0->initialize(v2, &rc.faces[f]);
        e1->initialize(v0, &rc.faces[f]);
        e2->initialize(v1, &rc.faces[f]);
        rc.faces[f].setEdges(e0, e1, e2);
    }
    for (int f = 0; f < nf; f++) rc.faces[f].update();

    std::vector<float> xf(x, x + 3 * nn), vf(v, v + 3 * nn), uf(u, u + 2 * nv);
    c->c.init(nn, xf.data(), vf.data(), nv, uf.data(), nf, fx, fu, nullptr, rc.mat->getDensity());
    // rest data from the reference's Face objects
    for (int f = 0; f < nf; f++) {
        const Face& F = rc.faces[f];
        c->c.finv[4 * f + 0] = F.inverse(0, 0);
        c->c.finv[4 * f + 1] = F.inverse(0, 1);
        c->c.finv[4 * f + 2] = F.inverse(1, 0);
        c->c.finv[4 * f + 3] = F.inverse(1, 1);
        c->c.farea[f] = F.area;
        c->c.fmass[f] = F.mass;
    }
    c->c.updateGeometry();
    RefClothImpl* self = c;
    c->c.syncHook = [self](orc::Cloth<float>& cl) {
        RefCloth& r = self->rc;
        for (size_t i = 0; i < r.nodes.size(); i++) {
            r.nodes[i].x = Vector3f(cl.x[3 * i], cl.x[3 * i + 1], cl.x[3 * i + 2]);
            r.nodes[i].v = Vector3f(cl.v[3 * i], cl.v[3 * i + 1], cl.v[3 * i + 2]);
            r.nodes[i].mass = cl.mass[i];
        }
        for (size_t f = 0; f < r.faces.size(); f++) {
            r.faces[f].update();
            for (int k = 0; k < 3; k++) cl.fn[3 * f + k] = r.faces[f].n(k);
        }
    };
    c->c.faceHook = [self](int f, float* fo, float* J) {
        Vector9f ff;
        Matrix9x9f JJ;
        stretchingForce(&self->rc.faces[f], self->rc.mat, ff, JJ);
        for (int p = 0; p < 9; p++) {
            fo[p] = ff(p);
            for (int q = 0; q < 9; q++) J[9 * p + q] = JJ(p, q);
        }
    };
    c->c.edgeHook = [self](int e, float* fo, float* J, float* theta) {
        Vector12f ff;
        Matrix12x12f JJ;
        bendingForce(&self->rc.edges[e], self->rc.mat, ff, JJ);
        for (int p = 0; p < 12; p++) {
            fo[p] = ff(p);
            for (int q = 0; q < 12; q++) J[12 * p + q] = JJ(p, q);
        }
        if (theta) *theta = self->rc.edges[e].angle();
    };
    // The reference's impulseForce and frictionForce (PhysicsHelper.cu:398-432) on a Proximity
    // whose nodes are this cloth's reference Nodes or, for points outside the cloth, Nodes
    // built from the given position, velocity, mass and free flag.
    c->c.proxHook = [self](int p, float d, float thickness, float dt, float* fI, float* JI, float* fF, float* JF) {
        const orc::ProximityRec<float>& pr = self->c.prox[p];
        Node ext[4];
        Proximity prox;
        for (int i = 0; i < 4; i++) {
            if (pr.node[i] >= 0) {
                prox.nodes[i] = &self->rc.nodes[pr.node[i]];
            } else {
                ext[i] = Node(Vector3f(pr.x[i][0], pr.x[i][1], pr.x[i][2]), ((pr.freeMask >> i) & 1) != 0);
                ext[i].v = Vector3f(pr.v[i][0], pr.v[i][1], pr.v[i][2]);
                ext[i].mass = pr.mass[i];
                prox.nodes[i] = &ext[i];
            }
            prox.w[i] = pr.w[i];
        }
        prox.n = Vector3f(pr.n[0], pr.n[1], pr.n[2]);
        prox.mu = pr.mu;
        prox.stiffness = pr.stiffness;
        Vector12f f;
        Matrix12x12f J;
        impulseForce(prox, d, thickness, f, J);
        for (int q = 0; q < 12; q++) {
            fI[q] = f(q);
            for (int k = 0; k < 12; k++) JI[12 * q + k] = J(q, k);
        }
        frictionForce(prox, d, thickness, dt, f, J);
        for (int q = 0; q < 12; q++) {
            fF[q] = f(q);
            for (int k = 0; k < 12; k++) JF[12 * q + k] = J(q, k);
        }
    };
    c->c.syncHook(c->c);
    return static_cast<ClothBase*>(c);
}

// Number of edges whose sides as set by the reference's Edge::initialize disagree with
// the oracle's restated topology (0 when the restatement is faithful).
int ref_cloth_topology_mismatches(void* cb) {
    auto* c = static_cast<RefClothImpl*>(static_cast<ClothBase*>(cb));
    const RefCloth& r = c->rc;
    const orc::Topology& t = c->c.topo;
    int bad = 0;
    for (int e = 0; e < t.nEdges(); e++) {
        const Edge& E = r.edges[e];
        for (int s = 0; s < 2; s++) {
            int face = E.adjacents[s] ? (int)(E.adjacents[s] - r.faces.data()) : -1;
            int opp = E.opposites[s] ? (int)(E.opposites[s] - r.verts.data()) : -1;
            int v0 = E.vertices[s][0] ? (int)(E.vertices[s][0] - r.verts.data()) : -1;
            int v1 = E.vertices[s][1] ? (int)(E.vertices[s][1] - r.verts.data()) : -1;
            if (face != t.eFace[2 * e + s] || opp != t.eOpp[2 * e + s] || v0 != t.eVert[4 * e + 2 * s] ||
                v1 != t.eVert[4 * e + 2 * s + 1])
                bad++;
        }
    }
    return bad;
}

}  // extern "C"

// Proximity detection through the reference's own signedVertexFaceDistance and
// signedEdgeEdgeDistance (MathHelper.cu:38-69), inEdge (PhysicsHelper.cu:3-18) and Proximity
// constructors (Proximity.cu:5-21), on each cloth's reference Node, Face and Edge objects
// (face normals by Face::update, edge areas by Edge::area).  Node normals and areas are the
// oracle's restatement of Mesh::updateNodeGeometries (Mesh.cu:182-203): Mesh.cu, which holds
// it, needs the renderer and is not compiled here.
static void orcDetectHooks(orc::Detector& D, const std::vector<ClothBase*>& cloths, const orc::DetectScene& S) {
    struct Span {
        RefClothImpl* c;
        int n0, f0, e0;
    };
    auto spans = std::make_shared<std::vector<Span>>();
    int n0 = 0, f0 = 0, e0 = 0;
    for (ClothBase* b : cloths) {
        auto* c = static_cast<RefClothImpl*>(b);
        c->c.syncHook(c->c);  // state into the reference objects, Face::update
        RefCloth& r = c->rc;
        for (size_t i = 0; i < r.nodes.size(); i++) {
            r.nodes[i].n = Vector3f(S.nn[3 * (n0 + i)], S.nn[3 * (n0 + i) + 1], S.nn[3 * (n0 + i) + 2]);
            r.nodes[i].area = S.narea[n0 + i];
        }
        spans->push_back({c, n0, f0, e0});
        n0 += (int)r.nodes.size();
        f0 += (int)r.faces.size();
        e0 += (int)r.edges.size();
    }
    auto find = [spans](int id, int Span::*off) -> const Span& {
        size_t k = 0;
        while (k + 1 < spans->size() && (*spans)[k + 1].*off <= id) k++;
        return (*spans)[k];
    };
    auto node = [find](int id) { const Span& s = find(id, &Span::n0); return &s.c->rc.nodes[id - s.n0]; };
    auto face = [find](int id) { const Span& s = find(id, &Span::f0); return &s.c->rc.faces[id - s.f0]; };
    auto edge = [find](int id) { const Span& s = find(id, &Span::e0); return &s.c->rc.edges[id - s.e0]; };
    auto sceneId = [spans](const Node* p) {
        for (const Span& s : *spans) {
            const std::vector<Node>& v = s.c->rc.nodes;
            if (p >= v.data() && p < v.data() + v.size()) return s.n0 + (int)(p - v.data());
        }
        return -1;
    };
    auto copyOut = [](const Vector3f& n, const float* w, orc::V3<float>& no, float* wo) {
        for (int c = 0; c < 3; c++) no[c] = n(c);
        for (int i = 0; i < 4; i++) wo[i] = w[i];
    };
    D.vfHook = [=](int nd, int fc, orc::V3<float>& n, float* w, float& h) {
        const Face* f = face(fc);
        Vector3f nn;
        float ww[4] = {0.f, 0.f, 0.f, 0.f};
        h = signedVertexFaceDistance(node(nd)->x, f->vertices[0]->node->x, f->vertices[1]->node->x,
                                     f->vertices[2]->node->x, nn, ww);
        if (std::isinf(h)) return false;
        copyOut(nn, ww, n, w);
        return true;
    };
    D.eeHook = [=](int a, int b, orc::V3<float>& n, float* w, float& h) {
        const Edge* ea = edge(a);
        const Edge* eb = edge(b);
        Vector3f nn;
        float ww[4] = {0.f, 0.f, 0.f, 0.f};
        h = signedEdgeEdgeDistance(ea->nodes[0]->x, ea->nodes[1]->x, eb->nodes[0]->x, eb->nodes[1]->x, nn, ww);
        if (std::isinf(h)) return false;
        copyOut(nn, ww, n, w);
        return true;
    };
    D.inEdgeHook = [=](float w, int a, int b) { return inEdge(w, edge(a), edge(b)); };
    auto fill = [=](const Proximity& p, orc::DetectedProximity& r) {
        for (int i = 0; i < 4; i++) {
            r.nodes[i] = sceneId(p.nodes[i]);
            r.w[i] = p.w[i];
        }
        for (int c = 0; c < 3; c++) r.n[c] = p.n(c);
        r.mu = p.mu;
        r.stiffness = p.stiffness;
    };
    D.proxVFHook = [=](int nd, int fc, const orc::DetectParams& P, orc::DetectedProximity& r) {
        fill(Proximity(node(nd), face(fc), P.collisionStiffness, P.clothFriction, 0.3f), r);
    };
    D.proxEEHook = [=](int a, int b, const orc::DetectParams& P, orc::DetectedProximity& r) {
        fill(Proximity(edge(a), edge(b), P.collisionStiffness, P.clothFriction, 0.3f), r);
    };
}

// Collision step parts through the reference's own code: checkVertexFaceImpact and
// checkEdgeEdgeImpact (CollisionHelper.cu:112-136, with checkImpact and its cubic solver) on
// the cloths' reference Node/Face/Edge objects, and CollisionOptimization (CPU branch of
// Optimization::solve, Optimization.cu:94-137) over reference Impacts.  The reference orders
// the optimization's nodes by address (the memory pool's allocation order, cloth by cloth),
// so the optimization runs on copies of the scene's nodes laid out in scene order.
static void orcCollideHooks(orc::Collider& K, const std::vector<ClothBase*>& cloths, orc::CollideScene& S) {
    struct Span {
        RefClothImpl* c;
        int n0, f0, e0;
        std::vector<int> nodeVert;  // a uv vertex of each node
    };
    auto spans = std::make_shared<std::vector<Span>>();
    int n0 = 0, f0 = 0, e0 = 0;
    for (ClothBase* b : cloths) {
        auto* c = static_cast<RefClothImpl*>(b);
        RefCloth& r = c->rc;
        Span sp{c, n0, f0, e0, std::vector<int>(r.nodes.size(), -1)};
        for (size_t i = 0; i < r.nodes.size(); i++) {
            Node& nd = r.nodes[i];
            nd.x = Vector3f(S.S.x[3 * (n0 + i)], S.S.x[3 * (n0 + i) + 1], S.S.x[3 * (n0 + i) + 2]);
            nd.x0 = Vector3f(S.x0[3 * (n0 + i)], S.x0[3 * (n0 + i) + 1], S.x0[3 * (n0 + i) + 2]);
            nd.x1 = nd.x;  // Mesh::updateNodeGeometries after the physics step (Mesh.cu:185)
            nd.mass = S.mass[n0 + i];
            nd.isFree = true;
        }
        for (size_t f = 0; f < r.faces.size(); f++)
            for (int k = 0; k < 3; k++) {
                const Vertex* v = r.faces[f].vertices[k];
                sp.nodeVert[v->node - r.nodes.data()] = (int)(v - r.verts.data());
            }
        spans->push_back(std::move(sp));
        n0 += (int)r.nodes.size();
        f0 += (int)r.faces.size();
        e0 += (int)r.edges.size();
    }
    auto find = [spans](int id, int Span::*off) -> const Span& {
        size_t k = 0;
        while (k + 1 < spans->size() && (*spans)[k + 1].*off <= id) k++;
        return (*spans)[k];
    };
    auto sceneId = [spans](const Node* p) {
        for (const Span& s : *spans) {
            const std::vector<Node>& v = s.c->rc.nodes;
            if (p >= v.data() && p < v.data() + v.size()) return s.n0 + (int)(p - v.data());
        }
        return -1;
    };
    auto nodePtr = [find](int id) {
        const Span& s = find(id, &Span::n0);
        return &s.c->rc.nodes[id - s.n0];
    };
    K.impactHook = [=](int type, int a, int b, float thickness, orc::Impact& imp) {
        ::Impact r;
        bool hit;
        if (type == 0) {
            const Span& sn = find(a, &Span::n0);
            const Span& sf = find(b, &Span::f0);
            const Vertex* v = &sn.c->rc.verts[sn.nodeVert[a - sn.n0]];
            hit = checkVertexFaceImpact(v, &sf.c->rc.faces[b - sf.f0], thickness, r);
        } else {
            const Span& s0 = find(a, &Span::e0);
            const Span& s1 = find(b, &Span::e0);
            hit = checkEdgeEdgeImpact(&s0.c->rc.edges[a - s0.e0], &s1.c->rc.edges[b - s1.e0], thickness, r);
        }
        if (!hit) return false;
        imp.type = type;
        imp.t = r.t;
        for (int k = 0; k < 4; k++) {
            imp.nodes[k] = sceneId(r.nodes[k]);
            imp.w[k] = r.w[k];
        }
        for (int k = 0; k < 3; k++) imp.n[k] = r.n(k);
        return true;
    };
    const int nTotal = n0;
    K.optimizeHook = [=](const std::vector<orc::Impact>& imps, float thickness, std::vector<float>& x) {
        std::vector<Node> scene(nTotal);  // node copies in scene order
        for (int id = 0; id < nTotal; id++) scene[id] = *nodePtr(id);
        std::vector<::Impact> ref(imps.size());
        for (size_t i = 0; i < imps.size(); i++) {
            for (int k = 0; k < 4; k++) {
                ref[i].nodes[k] = &scene[imps[i].nodes[k]];
                ref[i].w[k] = imps[i].w[k];
            }
            ref[i].t = imps[i].t;
            ref[i].n = Vector3f(imps[i].n[0], imps[i].n[1], imps[i].n[2]);
        }
        CollisionOptimization opt(ref, thickness, 0, 1e3f);
        opt.solve();
        for (int id = 0; id < nTotal; id++) {
            nodePtr(id)->x = scene[id].x;
            for (int c = 0; c < 3; c++) x[3 * id + c] = scene[id].x(c);
        }
    };
}
