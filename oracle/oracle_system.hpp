// CPU restatement of ClothSimulator's implicit step for one cloth: mesh topology
// (Mesh::load, CPU branch), assembly (Cloth::initializeForces / addExternalForces /
// addInternalForces / addHandleForces), the linear solve, and the step boundary
// (v += dv, Mesh::updatePositions, geometry refresh).
//
// TEST ORACLE ONLY: used by oracle/oracle.cpp, oracle/ref_adapter.cu, the tests and
// the CPU-baseline leg of bench.py, never by the product library.
#ifndef CLOTHSTEP_ORACLE_SYSTEM_HPP
#define CLOTHSTEP_ORACLE_SYSTEM_HPP

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <unordered_map>
#include <vector>

#include "oracle_math.hpp"
#include "sparse_chol.hpp"

namespace orc {

// Topology of one cloth, following Mesh::load (Mesh.cu:306-404) and Edge::initialize
// (Edge.cu:13-31).  Edges are numbered in order of first appearance while walking faces
// and their corners (v0v1, v1v2, v2v0), with nodes[0] < nodes[1] (Mesh.cu:56-68).
struct Topology {
    int nNodes = 0, nVerts = 0, nFaces = 0;
    std::vector<int> fx, fu;  // 3 per face: node index and uv-vertex index of each corner
    // Edge e: nodes[2]; for side s in {0,1}: face (-1 if none), uv vertices [s][0], [s][1]
    // (vertices[s][0] belongs to nodes[0]) and the opposite uv vertex.
    std::vector<int> eNodes, eFace, eVert, eOpp;
    int nEdges() const { return (int)eNodes.size() / 2; }
    bool interior(int e) const { return eFace[2 * e] >= 0 && eFace[2 * e + 1] >= 0; }

    void build(int nn, int nv, int nf, const int* fxIn, const int* fuIn) {
        nNodes = nn; nVerts = nv; nFaces = nf;
        fx.assign(fxIn, fxIn + 3 * nf);
        fu.assign(fuIn, fuIn + 3 * nf);
        eNodes.clear(); eFace.clear(); eVert.clear(); eOpp.clear();
        std::unordered_map<uint64_t, int> map;
        map.reserve(3 * nf);
        auto find = [&](int a, int b) {
            if (a > b) std::swap(a, b);
            uint64_t key = (uint64_t)(uint32_t)a << 32 | (uint32_t)b;
            auto it = map.find(key);
            if (it != map.end()) return it->second;
            int id = (int)eNodes.size() / 2;
            map[key] = id;
            eNodes.push_back(a); eNodes.push_back(b);
            eFace.push_back(-1); eFace.push_back(-1);
            for (int i = 0; i < 4; i++) eVert.push_back(-1);
            eOpp.push_back(-1); eOpp.push_back(-1);
            return id;
        };
        auto init = [&](int e, int oppCorner, int f) {
            for (int i = 0; i < 3; i++) {
                int c0 = i, c1 = (i + 1) % 3;
                int n0 = fx[3 * f + c0], n1 = fx[3 * f + c1];
                if (eNodes[2 * e] == n0 && eNodes[2 * e + 1] == n1) {
                    eVert[4 * e + 0] = fu[3 * f + c0];
                    eVert[4 * e + 1] = fu[3 * f + c1];
                    eOpp[2 * e] = fu[3 * f + oppCorner];
                    eFace[2 * e] = f;
                    return;
                } else if (eNodes[2 * e + 1] == n0 && eNodes[2 * e] == n1) {
                    eVert[4 * e + 2] = fu[3 * f + c1];
                    eVert[4 * e + 3] = fu[3 * f + c0];
                    eOpp[2 * e + 1] = fu[3 * f + oppCorner];
                    eFace[2 * e + 1] = f;
                    return;
                }
            }
        };
        for (int f = 0; f < nf; f++) {
            int a = fx[3 * f], b = fx[3 * f + 1], c = fx[3 * f + 2];
            int e0 = find(a, b), e1 = find(b, c), e2 = find(c, a);
            init(e0, 2, f);
            init(e1, 0, f);
            init(e2, 1, f);
        }
    }
};

// uv-vertex -> node map, as Vertex::node is set at Mesh.cu:388-390.
inline std::vector<int> vertexNodes(const Topology& t) {
    std::vector<int> vn(t.nVerts, -1);
    for (int f = 0; f < t.nFaces; f++)
        for (int c = 0; c < 3; c++) vn[t.fu[3 * f + c]] = t.fx[3 * f + c];
    return vn;
}

struct StepParams {
    double dt;
    double gravity[3];
    double windDensity, windDrag, windVelocity[3];
    double handleStiffness;
};

// One proximity as Cloth::physicsStep receives it (Proximity.cuh:11-21).  node[i] >= 0: a
// node of this cloth (its x, v, mass are the cloth's; cloth nodes are free, Mesh.cu:349);
// node[i] < 0: a point outside the cloth (another cloth's node or an obstacle's) with the
// given x, v, mass and free flag (bit i of freeMask); its rows and columns are skipped, as
// Cloth.cu:176-177 marks nodes the mesh does not contain with index -1.
template <class T>
struct ProximityRec {
    int node[4];
    T x[4][3], v[4][3], mass[4];
    int freeMask;
    T n[3], w[4], mu, stiffness;
};

// Sparse block accumulator with the reference's accumulation order: one float (or
// double) per scalar entry, updated element by element in mesh order exactly like
// Eigen's coeffRef(i,j) += v (Cloth.cu:42-76).  The pattern is fixed per mesh.
template <class T>
struct BlockSystem {
    int n = 0;                        // nodes
    std::vector<int> rowPtr, col;     // block CSR (sorted columns)
    std::vector<T> val;               // 9 per block, row-major within a block
    std::vector<T> b;                 // 3n
    int find(int i, int j) const {
        const int* lo = col.data() + rowPtr[i];
        const int* hi = col.data() + rowPtr[i + 1];
        const int* p = std::lower_bound(lo, hi, j);
        return (int)(p - col.data());
    }
};

template <class T>
struct Cloth {
    Topology topo;
    std::vector<int> vnode;
    const Material<T>* mat = nullptr;  // restated material; unused when the hooks below are set
    T density = T(0);
    // Optional replacements of the element evaluation and of the per-assembly state sync,
    // used by the reference adapter to call the reference's own functions.
    std::function<void(Cloth&)> syncHook;
    std::function<void(int, T*, T*)> faceHook;
    std::function<void(int, T*, T*, T*)> edgeHook;
    // (proximity, depth, thickness, dt, impulse f, J, friction f, J)
    std::function<void(int, T, T, T, T*, T*, T*, T*)> proxHook;
    std::vector<ProximityRec<T>> prox;
    T proxThickness = T(0);
    std::vector<T> x, v, u;           // 3N, 3N, 2U
    std::vector<T> x0;                // positions at the start of the last step (Node::x0)
    std::vector<T> finv, farea, fmass, fn;  // per face: 4, 1, 1, 3 (normal)
    std::vector<T> mass;              // per node
    std::vector<int> handleNode;
    std::vector<T> handlePos;         // 3 per handle
    BlockSystem<T> sys;

    void init(int nn, const T* xIn, const T* vIn, int nv, const T* uIn, int nf, const int* fxIn, const int* fuIn,
              const Material<T>* m, T dens) {
        mat = m;
        density = dens;
        topo.build(nn, nv, nf, fxIn, fuIn);
        vnode = vertexNodes(topo);
        x.assign(xIn, xIn + 3 * nn);
        x0 = x;  // Node::Node (Node.cu:5-11)
        v.assign(vIn, vIn + 3 * nn);
        u.assign(uIn, uIn + 2 * nv);
        finv.resize(4 * nf); farea.resize(nf); fmass.resize(nf); fn.resize(3 * nf);
        for (int f = 0; f < nf; f++) {
            T inv[2][2], area;
            faceRest<T>(&u[2 * topo.fu[3 * f]], &u[2 * topo.fu[3 * f + 1]], &u[2 * topo.fu[3 * f + 2]], inv, area);
            finv[4 * f + 0] = inv[0][0]; finv[4 * f + 1] = inv[0][1];
            finv[4 * f + 2] = inv[1][0]; finv[4 * f + 3] = inv[1][1];
            farea[f] = area;
            fmass[f] = area * density;  // Face.cu:18
        }
        updateGeometry();
        buildPattern();
    }

    V3<T> X(int i) const { return v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]); }
    V3<T> Vel(int i) const { return v3(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }
    V3<T> N(int f) const { return v3(fn[3 * f], fn[3 * f + 1], fn[3 * f + 2]); }

    // Face normals (Face.cu:124-132; free faces keep their rest area) and node masses
    // (Mesh.cu:182-203: lumped mass = sum of face.mass/3 in face order).
    void updateGeometry() {
        int nf = topo.nFaces;
        for (int f = 0; f < nf; f++) {
            V3<T> n = faceNormal(X(topo.fx[3 * f]), X(topo.fx[3 * f + 1]), X(topo.fx[3 * f + 2]));
            for (int c = 0; c < 3; c++) fn[3 * f + c] = n[c];
        }
        mass.assign(topo.nNodes, T(0));
        for (int f = 0; f < nf; f++) {
            T m = fmass[f] / T(3);
            for (int c = 0; c < 3; c++) mass[topo.fx[3 * f + c]] += m;
        }
    }

    void buildPattern() {
        int n = topo.nNodes;
        std::vector<std::vector<int>> adj(n);
        for (int i = 0; i < n; i++) adj[i].push_back(i);
        auto link = [&](const int* ids, int k) {
            for (int a = 0; a < k; a++)
                for (int b = 0; b < k; b++) adj[ids[a]].push_back(ids[b]);
        };
        for (int f = 0; f < topo.nFaces; f++) link(&topo.fx[3 * f], 3);
        for (int e = 0; e < topo.nEdges(); e++)
            if (topo.interior(e)) {
                int ids[4];
                edgeNodes(e, ids);
                link(ids, 4);
            }
        // proximity pairs enter the pattern as Eigen's coeffRef inserts them
        for (const ProximityRec<T>& pr : prox)
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++)
                    if (pr.node[a] >= 0 && pr.node[b] >= 0) adj[pr.node[a]].push_back(pr.node[b]);
        sys.n = n;
        sys.rowPtr.assign(n + 1, 0);
        sys.col.clear();
        for (int i = 0; i < n; i++) {
            std::sort(adj[i].begin(), adj[i].end());
            adj[i].erase(std::unique(adj[i].begin(), adj[i].end()), adj[i].end());
            sys.rowPtr[i + 1] = sys.rowPtr[i] + (int)adj[i].size();
            sys.col.insert(sys.col.end(), adj[i].begin(), adj[i].end());
        }
        sys.val.assign(9 * sys.col.size(), T(0));
        sys.b.assign(3 * n, T(0));
    }

    // nodes[0], nodes[1], opposite node of side 0, opposite node of side 1
    // (PhysicsHelper.cu:363-368).
    void edgeNodes(int e, int ids[4]) const {
        ids[0] = topo.eNodes[2 * e];
        ids[1] = topo.eNodes[2 * e + 1];
        ids[2] = vnode[topo.eOpp[2 * e]];
        ids[3] = vnode[topo.eOpp[2 * e + 1]];
    }

    void faceForce(int f, T fo[9], T J[81]) const {
        if (faceHook) { faceHook(f, fo, J); return; }
        T inv[2][2] = {{finv[4 * f], finv[4 * f + 1]}, {finv[4 * f + 2], finv[4 * f + 3]}};
        stretchingForce<T>(*mat, X(topo.fx[3 * f]), X(topo.fx[3 * f + 1]), X(topo.fx[3 * f + 2]), inv, farea[f], fo, J);
    }

    void edgeForce(int e, T fo[12], T J[144], T* theta = nullptr) const {
        if (edgeHook) { edgeHook(e, fo, J, theta); return; }
        int ids[4];
        edgeNodes(e, ids);
        int f0 = topo.eFace[2 * e], f1 = topo.eFace[2 * e + 1];
        T area = farea[f0] + farea[f1];
        const int* ev = &topo.eVert[4 * e];
        T d0[2] = {u[2 * ev[1]] - u[2 * ev[0]], u[2 * ev[1] + 1] - u[2 * ev[0] + 1]};
        T d1[2] = {u[2 * ev[3]] - u[2 * ev[2]], u[2 * ev[3] + 1] - u[2 * ev[2] + 1]};
        bendingForce<T>(*mat, X(ids[0]), X(ids[1]), X(ids[2]), X(ids[3]), N(f0), N(f1), area, d0, d1, fo, J, theta);
    }

    // Sets the proximities of the next steps (rebuilds the pattern).
    void setProximities(const std::vector<ProximityRec<T>>& recs, T thickness) {
        prox = recs;
        proxThickness = thickness;
        buildPattern();
    }

    // Position, velocity of a proximity's node i (Cloth.cu:174, 180-181).
    V3<T> proxX(const ProximityRec<T>& pr, int i) const {
        return pr.node[i] >= 0 ? X(pr.node[i]) : v3(pr.x[i][0], pr.x[i][1], pr.x[i][2]);
    }
    V3<T> proxV(const ProximityRec<T>& pr, int i) const {
        return pr.node[i] >= 0 ? Vel(pr.node[i]) : v3(pr.v[i][0], pr.v[i][1], pr.v[i][2]);
    }

    // Depth and the impulse and friction forces and Jacobians of proximity p at the current
    // state (Cloth.cu:179-190).
    T proximityForces(int p, T dt, T fI[12], T JI[144], T fF[12], T JF[144]) const {
        const ProximityRec<T>& pr = prox[p];
        V3<T> xs[4], vs[4];
        T ms[4];
        int freeMask = 0;
        for (int i = 0; i < 4; i++) {
            xs[i] = proxX(pr, i);
            vs[i] = proxV(pr, i);
            ms[i] = pr.node[i] >= 0 ? mass[pr.node[i]] : pr.mass[i];
            if (pr.node[i] >= 0 || (pr.freeMask & (1 << i))) freeMask |= 1 << i;
        }
        const V3<T> n = v3(pr.n[0], pr.n[1], pr.n[2]);
        const T d = proximityDepth<T>(pr.w, n, xs, proxThickness);
        if (proxHook) {
            proxHook(p, d, proxThickness, dt, fI, JI, fF, JF);
            return d;
        }
        impulseForce<T>(pr.w, n, pr.stiffness, d, proxThickness, fI, JI);
        frictionForce<T>(pr.w, n, pr.mu, pr.stiffness, d, proxThickness, dt, vs, ms, freeMask, fF, JF);
        return d;
    }

    // Cloth.cu:42-76 with rows and columns of index -1 skipped.
    void addElementSkip(const T* B, const T* bb, const int* ids) {
        for (int i = 0; i < 4; i++) {
            int xi = ids[i];
            if (xi < 0) continue;
            for (int j = 0; j < 4; j++) {
                if (ids[j] < 0) continue;
                int blk = sys.find(xi, ids[j]);
                for (int k = 0; k < 3; k++)
                    for (int h = 0; h < 3; h++) sys.val[9 * blk + 3 * k + h] += B[(3 * i + k) * 12 + 3 * j + h];
            }
            for (int j = 0; j < 3; j++) sys.b[3 * xi + j] += bb[3 * i + j];
        }
    }

    template <int K>
    void addElement(const T* B, const T* bb, const int* ids) {
        // Cloth.cu:42-76: A(3x+k, 3y+h) += B(3i+k, 3j+h); b(3x+j) += bb(3i+j).
        for (int i = 0; i < K; i++) {
            int xi = ids[i];
            for (int j = 0; j < K; j++) {
                int blk = sys.find(xi, ids[j]);
                for (int k = 0; k < 3; k++)
                    for (int h = 0; h < 3; h++) sys.val[9 * blk + 3 * k + h] += B[(3 * i + k) * (3 * K) + 3 * j + h];
            }
            for (int j = 0; j < 3; j++) sys.b[3 * xi + j] += bb[3 * i + j];
        }
    }

    // -dt*dt*J and dt*(f + dt*J*v) for one element (Cloth.cu:137, 153).
    template <int K>
    static void elementSystem(T dt, const T* f, const T* J, const T* vel, T* B, T* bb) {
        const int n = 3 * K;
        T s = -dt * dt;
        for (int p = 0; p < n * n; p++) B[p] = s * J[p];
        for (int p = 0; p < n; p++) {
            T jv = T(0);
            for (int q = 0; q < n; q++) jv += (dt * J[p * n + q]) * vel[q];
            bb[p] = dt * (f[p] + jv);
        }
    }

    // Full assembly in the reference order (Cloth.cu:676-684).
    void assemble(const StepParams& P) {
        const T dt = (T)P.dt;
        int n = topo.nNodes;
        if (syncHook) syncHook(*this);
        std::fill(sys.val.begin(), sys.val.end(), T(0));
        std::fill(sys.b.begin(), sys.b.end(), T(0));
        // initializeForces: A = diag(mass) (Cloth.cu:78-92)
        for (int i = 0; i < n; i++) {
            int blk = sys.find(i, i);
            for (int j = 0; j < 3; j++) sys.val[9 * blk + 4 * j] = mass[i];
        }
        // addExternalForces: gravity then wind (Cloth.cu:94-123)
        V3<T> g = v3((T)P.gravity[0], (T)P.gravity[1], (T)P.gravity[2]);
        for (int i = 0; i < n; i++) {
            V3<T> gi = scl(dt * mass[i], g);
            for (int j = 0; j < 3; j++) sys.b[3 * i + j] += gi[j];
        }
        V3<T> wv = v3((T)P.windVelocity[0], (T)P.windVelocity[1], (T)P.windVelocity[2]);
        T wden = (T)P.windDensity, wdrag = (T)P.windDrag;
        for (int f = 0; f < topo.nFaces; f++) {
            V3<T> nrm = N(f);
            T area = farea[f];
            int a = topo.fx[3 * f], b = topo.fx[3 * f + 1], c = topo.fx[3 * f + 2];
            V3<T> avg = dvd(add(add(Vel(a), Vel(b)), Vel(c)), T(3));
            V3<T> rel = sub(wv, avg);
            T vn = dot(nrm, rel);
            V3<T> vt = sub(rel, scl(vn, nrm));
            V3<T> force = dvd(scl(area, add(scl(wden * ab(vn) * vn, nrm), scl(wdrag, vt))), T(3));
            V3<T> fo = scl(dt, force);
            for (int j = 0; j < 3; j++) {
                sys.b[3 * a + j] += fo[j];
                sys.b[3 * b + j] += fo[j];
                sys.b[3 * c + j] += fo[j];
            }
        }
        // addInternalForces: faces, then interior edges (Cloth.cu:125-155)
        T fo[12], J[144], B[144], bb[12], vel[12];
        for (int f = 0; f < topo.nFaces; f++) {
            faceForce(f, fo, J);
            const int* ids = &topo.fx[3 * f];
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) vel[3 * a + c] = v[3 * ids[a] + c];
            elementSystem<3>(dt, fo, J, vel, B, bb);
            addElement<3>(B, bb, ids);
        }
        for (int e = 0; e < topo.nEdges(); e++) {
            if (!topo.interior(e)) continue;
            int ids[4];
            edgeNodes(e, ids);
            edgeForce(e, fo, J);
            for (int a = 0; a < 4; a++)
                for (int c = 0; c < 3; c++) vel[3 * a + c] = v[3 * ids[a] + c];
            elementSystem<4>(dt, fo, J, vel, B, bb);
            addElement<4>(B, bb, ids);
        }
        // addHandleForces (Cloth.cu:157-169)
        T k = (T)P.handleStiffness;
        for (size_t h = 0; h < handleNode.size(); h++) {
            int i = handleNode[h];
            int blk = sys.find(i, i);
            for (int j = 0; j < 3; j++) sys.val[9 * blk + 4 * j] += dt * dt * k;
            V3<T> p = v3(handlePos[3 * h], handlePos[3 * h + 1], handlePos[3 * h + 2]);
            V3<T> fh = mul(scl(dt, sub(sub(p, X(i)), scl(dt, Vel(i)))), k);
            for (int j = 0; j < 3; j++) sys.b[3 * i + j] += fh[j];
        }
        // addProximityForces (Cloth.cu:171-192): per proximity, the impulse term
        // (-dt^2 J, dt (f + dt J v)) then the friction term (-dt J, dt f)
        for (size_t pi = 0; pi < prox.size(); pi++) {
            const ProximityRec<T>& pr = prox[pi];
            T fI[12], JI[144], fF[12], JF[144];
            proximityForces((int)pi, dt, fI, JI, fF, JF);
            for (int a = 0; a < 4; a++) {
                V3<T> va = proxV(pr, a);
                for (int c = 0; c < 3; c++) vel[3 * a + c] = va[c];
            }
            elementSystem<4>(dt, fI, JI, vel, B, bb);
            addElementSkip(B, bb, pr.node);
            const T sF = -dt;
            for (int q = 0; q < 144; q++) B[q] = sF * JF[q];
            for (int q = 0; q < 12; q++) bb[q] = dt * fF[q];
            addElementSkip(B, bb, pr.node);
        }
    }

    // v += dv (Cloth.cu:690-692); x0 = x, x += dt v (Mesh.cu:226-231); refresh geometry
    // (Simulator.cu:596-597).
    void advance(const T* dv, T dt) {
        int n = topo.nNodes;
        for (int i = 0; i < 3 * n; i++) v[i] += dv[i];
        x0 = x;
        for (int i = 0; i < 3 * n; i++) x[i] += dt * v[i];
        updateGeometry();
    }
};

// Expand a block system to scalar CSR (for the factorisation).
template <class T, class S>
inline void toScalarCsr(const BlockSystem<T>& s, std::vector<int>& rp, std::vector<int>& ci, std::vector<S>& vv) {
    int n = s.n;
    rp.assign(3 * n + 1, 0);
    ci.clear();
    vv.clear();
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            int r = 3 * i + k;
            for (int p = s.rowPtr[i]; p < s.rowPtr[i + 1]; p++)
                for (int h = 0; h < 3; h++) {
                    ci.push_back(3 * s.col[p] + h);
                    vv.push_back((S)s.val[9 * p + 3 * k + h]);
                }
            rp[r + 1] = (int)ci.size();
        }
}

// y = A x with a block system, accumulated in S.
template <class T, class S>
inline void blockSpmv(const BlockSystem<T>& s, const S* xin, S* y) {
    for (int i = 0; i < s.n; i++) {
        S acc[3] = {S(0), S(0), S(0)};
        for (int p = s.rowPtr[i]; p < s.rowPtr[i + 1]; p++) {
            int j = s.col[p];
            for (int k = 0; k < 3; k++)
                for (int h = 0; h < 3; h++) acc[k] += (S)s.val[9 * p + 3 * k + h] * xin[3 * j + h];
        }
        for (int k = 0; k < 3; k++) y[3 * i + k] = acc[k];
    }
}

// FP64 block-Jacobi preconditioned CG to a relative residual (oracle for large systems).
template <class T>
inline int blockJacobiPcg64(const BlockSystem<T>& s, const double* b, double* x, double relTol, int maxIter,
                            double* relRes) {
    int n = s.n, m = 3 * n;
    std::vector<double> Pinv(9 * n), r(m), z(m), p(m), q(m);
    for (int i = 0; i < n; i++) {
        int blk = s.find(i, i);
        double a[9];
        for (int t = 0; t < 9; t++) a[t] = s.val[9 * blk + t];
        double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
        double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
        double id = 1.0 / det;
        double* P = &Pinv[9 * i];
        P[0] = c00 * id; P[1] = (a[2] * a[7] - a[1] * a[8]) * id; P[2] = (a[1] * a[5] - a[2] * a[4]) * id;
        P[3] = c01 * id; P[4] = (a[0] * a[8] - a[2] * a[6]) * id; P[5] = (a[2] * a[3] - a[0] * a[5]) * id;
        P[6] = c02 * id; P[7] = (a[1] * a[6] - a[0] * a[7]) * id; P[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    }
    blockSpmv<T, double>(s, x, q.data());
    double bn = 0;
    for (int i = 0; i < m; i++) { r[i] = b[i] - q[i]; bn += b[i] * b[i]; }
    bn = std::sqrt(bn);
    if (bn == 0) bn = 1;
    auto prec = [&](const std::vector<double>& in, std::vector<double>& out) {
        for (int i = 0; i < n; i++)
            for (int k = 0; k < 3; k++)
                out[3 * i + k] = Pinv[9 * i + 3 * k] * in[3 * i] + Pinv[9 * i + 3 * k + 1] * in[3 * i + 1] +
                                 Pinv[9 * i + 3 * k + 2] * in[3 * i + 2];
    };
    prec(r, z);
    p = z;
    double rz = 0;
    for (int i = 0; i < m; i++) rz += r[i] * z[i];
    int it = 0;
    double rr = 0;
    for (int i = 0; i < m; i++) rr += r[i] * r[i];
    while (std::sqrt(rr) / bn > relTol && it < maxIter) {
        blockSpmv<T, double>(s, p.data(), q.data());
        double pq = 0;
        for (int i = 0; i < m; i++) pq += p[i] * q[i];
        double alpha = rz / pq;
        for (int i = 0; i < m; i++) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
        prec(r, z);
        double rz2 = 0;
        rr = 0;
        for (int i = 0; i < m; i++) { rz2 += r[i] * z[i]; rr += r[i] * r[i]; }
        double beta = rz2 / rz;
        rz = rz2;
        for (int i = 0; i < m; i++) p[i] = z[i] + beta * p[i];
        it++;
    }
    // true residual
    blockSpmv<T, double>(s, x, q.data());
    double tr = 0;
    for (int i = 0; i < m; i++) tr += (b[i] - q[i]) * (b[i] - q[i]);
    if (relRes) *relRes = std::sqrt(tr) / bn;
    return it;
}

}  // namespace orc

#endif
