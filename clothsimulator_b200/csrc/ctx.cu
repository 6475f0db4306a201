// Host runtime of the B200 implicit cloth step and its C ABI (include/clothstep.h).
//
// cs_load_batch turns a batch of cloths into the HBM layout of cs_internal.h:
//   * edges in the reference's numbering (first appearance while walking the faces'
//     corners, Mesh.cu:56-68, 385-395) with sides as Edge::initialize sets them
//     (Edge.cu:13-31); only interior edges carry bending (Cloth.cu:140-154);
//   * face rest data exactly as Face::initialize computes it (Face.cu:12-20), lumped node
//     masses as Mesh::updateNodeGeometries sums them (Mesh.cu:190-200);
//   * the fixed 3x3-block pattern of A (diagonal + face pairs + bending stencils) in SELL-32
//     slices, and for every block its contributors in the reference's accumulation order,
//     so the gather kernel reproduces Cloth::addMatrixAndVector's sums (Cloth.cu:42-76)
//     without atomics.  Pattern, columns and contributor lists are built once per distinct
//     topology and shared by every sheet that has it;
//   * the 30^3 stretching tables (Material.cu:28-36) per distinct material and multiplier.
// cs_step runs the whole step as one CUDA graph whose solve loop is a device-driven
// conditional while node (no host round trip per iteration, unlike Cloth.cu:784-809).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "../../include/clothstep.h"
#include "cs_internal.h"
#include "mlp.h"

// kernels (forces.cu, pcg.cu)
__global__ void cs_edge_kernel(Batch B);
__global__ void cs_gather_kernel(Batch B);
__global__ void cs_expand_kernel(Batch B, float* face_f, float* face_J, float* edge_f, float* edge_J);
__global__ void cs_reduce1_kernel(Batch B);
__global__ void cs_vector_kernel(Batch B);
__global__ void cs_reduce2_kernel(Batch B, cudaGraphConditionalHandle handle);
__global__ void cs_solve_prologue_kernel(Batch B);
__global__ void cs_solve_setup_kernel(Batch B);
__global__ void cs_advance_kernel(Batch B);
__global__ void cs_spmv_plain_kernel(Batch B, const float* x, float* y);
__global__ void cs_profile_setup_kernel(Batch B, int phase);
__global__ void cs_resident_pcg_kernel(Batch B);
__global__ void cs_coarse_setup_kernel(Batch B);
static_assert(CS_SPMV_CANDIDATES == CS_TUNE_SPMV_SHAPES, "the tuner's result holds every SpMV shape");
__global__ void cs_prox_kernel(Batch B);
__global__ void cs_prox_row_kernel(Batch B);
__global__ void cs_slice_bnorm_kernel(Batch B);
__global__ void cs_bc_assemble_kernel(Batch B);
__global__ void cs_bc_invert_small_kernel(Batch B);
__global__ void cs_bc_invert_cluster_kernel(Batch B);
__global__ void cs_bc_restrict_kernel(Batch B);
__global__ void cs_bc_apply_kernel(Batch B);
__global__ void cs_bc_finish_kernel(Batch B);
__global__ void cs_scan_sums_kernel(const int* data, int n, int* partial);
__global__ void cs_scan_partials_kernel(int* partial, int nb, int* total);
__global__ void cs_scan_apply_kernel(int* data, int n, const int* partial);
__global__ void cs_prox_count_kernel(Batch B, const cs_proximity_desc* d, int n, int* icount);
__global__ void cs_prox_expand_kernel(Batch B, const cs_proximity_desc* d, int n, const int* ioff, float thickness,
                                      ProxInst* inst, int* sheet_prox);
__global__ void cs_prox_rowcount_kernel(const ProxInst* inst, int T, int* rowCount);
__global__ void cs_prox_rowfill_kernel(const ProxInst* inst, int T, const int* rowPtr, int* rowFill, int* rowInst);
__global__ void cs_prox_rowsort_kernel(int N, const int* rowPtr, int* rowInst);
__global__ void cs_prox_outside_kernel(Batch B, const int* rowPtr, const int* rowInst, const ProxInst* inst,
                                       const int* xptr, int* out);
__global__ void cs_contact_face_kernel(Batch B, Contact C);
__global__ void cs_contact_node_kernel(Batch B, Contact C);
__global__ void cs_contact_grid_kernel(Batch B, Contact C, const int* sheet_group);
__global__ void cs_contact_pair_kernel(Batch B, Contact C, const int* sheet_group);
__global__ void cs_contact_vf_kernel(Batch B, Contact C, int npairs);
__global__ void cs_impact_kernel(Batch B, Contact C, Collide K, int npairs);
__global__ void cs_impact_keys_kernel(Collide K, int n, int pass, const int* perm, unsigned long long* key,
                                      int* perm_out);
__global__ void cs_impact_gather_kernel(Collide K, int n, const int* perm);
__global__ void cs_select_init_kernel(Collide K, int n);
__global__ void cs_select_reset_kernel(Collide K, int n);
__global__ void cs_select_min_kernel(Collide K, int n);
__global__ void cs_select_choose_kernel(Collide K, int n);
__global__ void cs_select_drop_kernel(Collide K, int n);
__global__ void cs_select_write_kernel(Collide K, int n, int base, int cap);
__global__ void cs_opt_mark_kernel(Collide K, int nc);
__global__ void cs_opt_nodes_kernel(Collide K, int N);
__global__ void cs_opt_idx_kernel(Collide K, int nc);
__global__ void cs_opt_fill_kernel(Collide K, int nc);
__global__ void cs_opt_sort_kernel(Collide K, int nn);
__global__ void cs_opt_kernel(Batch B, Collide K, int nn, int nc);
__global__ void cs_collide_velocity_kernel(Batch B, float invDt);
__global__ void cs_contact_ee_kernel(Batch B, Contact C, int npairs);
__global__ void cs_contact_count_kernel(Contact C);
__global__ void cs_contact_scan_kernel(Contact C, int nblocks);
__global__ void cs_contact_write_kernel(Batch B, Contact C);

namespace {

// ---------------------------------------------------------------------------------------
// Material tables (Material.cu:3-85), host side, float arithmetic in the reference's order.

void eigen2(float a, float b, float d, float Q[2][2], float l[2]) {  // MathHelper.cu:3-36
    float amd = a - d, apd = a + d, b2 = b * b;
    float det = std::sqrt(4.0f * b2 + amd * amd);
    float l1 = 0.5f * (apd + det), l2 = 0.5f * (apd - det);
    l[0] = l1;
    l[1] = l2;
    if (b != 0.0f) {
        float v0 = l1 - d, v1 = b, vn = std::sqrt(v0 * v0 + b2);
        Q[0][0] = v0 / vn;
        Q[1][0] = v1 / vn;
        v0 = l2 - d;
        vn = std::sqrt(v0 * v0 + b2);
        Q[0][1] = v0 / vn;
        Q[1][1] = v1 / vn;
    } else if (a >= d) {
        Q[0][0] = 1.0f; Q[1][0] = 0.0f; Q[0][1] = 0.0f; Q[1][1] = 1.0f;
    } else {
        Q[0][0] = 0.0f; Q[1][0] = 1.0f; Q[0][1] = 1.0f; Q[1][1] = 0.0f;
    }
}

float clampf(float x, float a, float b) { return x < a ? a : (x > b ? b : x); }

// calculateStretchingSample (Material.cu:45-85); data[2][5][4] as built at Material.cu:20-27.
void stretchingSample(float G00, float G01, float G11, const float data[2][5][4], float out[4]) {
    float Q[2][2], l[2];
    eigen2(2.0f * G00, 2.0f * G01, 2.0f * G11, Q, l);
    if (l[0] == l[1] && Q[0][0] == 0.0f && Q[1][1] == 0.0f) {
        Q[0][0] = 1.0f; Q[0][1] = 0.0f; Q[1][0] = 0.0f; Q[1][1] = 1.0f;
    }
    if (Q[0][0] < 0.0f) { Q[0][0] = -Q[0][0]; Q[1][0] = -Q[1][0]; }
    if (Q[1][1] < 0.0f) { Q[0][1] = -Q[0][1]; Q[1][1] = -Q[1][1]; }
    float strainWeight = (std::sqrt(l[0] + 1.0f) - 1.0f) * 6.0f;
    strainWeight = clampf(strainWeight, 0.0f, 1.0f - 1e-6f);
    int strainId = (int)strainWeight;
    strainWeight -= strainId;
    float q10 = Q[1][0], q00 = Q[0][0];
    float at = std::atan2(q10, q00);
    float angleWeight = (float)((double)(at < 0.0f ? -at : at) / M_PI * 8.0f);
    angleWeight = clampf(angleWeight, 0.0f, 4.0f - 1e-6f);
    int angleId = (int)angleWeight;
    angleWeight -= angleId;
    float w[2][2] = {{(1.0f - strainWeight) * (1.0f - angleWeight), (1.0f - strainWeight) * angleWeight},
                     {strainWeight * (1.0f - angleWeight), strainWeight * angleWeight}};
    float ans[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int c = 0; c < 4; c++) ans[c] += data[strainId + i][angleId + j][c] * w[i][j];
    for (int c = 0; c < 4; c++) out[c] = (ans[c] > 0.0f ? ans[c] : 0.0f) * 2.0f;
}

// Unscaled 30^3 samples of one material's stretching rows.
std::vector<float> stretchingSamples(const float rows[6][4]) {
    float data[2][5][4];
    for (int c = 0; c < 4; c++) data[0][0][c] = rows[0][c];
    for (int i = 1; i < 5; i++)
        for (int c = 0; c < 4; c++) data[0][i][c] = data[0][0][c];
    for (int i = 0; i < 5; i++)
        for (int c = 0; c < 4; c++) data[1][i][c] = rows[i + 1][c];
    std::vector<float> out(4 * CS_TABLE_ENTRIES);
    for (int i = 0; i < CS_TABLE_N; i++)
        for (int j = 0; j < CS_TABLE_N; j++)
            for (int k = 0; k < CS_TABLE_N; k++) {
                float G00 = (float)i / CS_TABLE_N - 0.25f;
                float G11 = (float)j / CS_TABLE_N - 0.25f;
                float G01 = (float)k / CS_TABLE_N;
                stretchingSample(G00, G01, G11, data, &out[4 * ((i * CS_TABLE_N + j) * CS_TABLE_N + k)]);
            }
    return out;
}

// Bias weight of one uv edge after the fold and clamp of Material.cu:130-133.
float biasWeight(float d0, float d1) {
    float at = std::atan2(d1, d0);
    float w = (float)((double)((at < 0.0f ? -at : at) * 4.0f) / M_PI);
    if (w > 2.0f) w = 4.0f - w;
    return clampf(w, 0.0f, 2.0f - 1e-6f);
}

// ---------------------------------------------------------------------------------------
// Topology and pattern of one distinct mesh connectivity.

struct Topo {
    int n_nodes = 0, n_verts = 0, n_faces = 0;
    std::vector<int> fx, fu;
    // interior edges in reference order
    std::vector<int> ie_nodes;  // 4 per: n0, n1, opposite node side 0, side 1
    std::vector<int> ie_faces;  // 2 per
    std::vector<int> ie_meta;   // rotations of the adjacent faces' vertex order
    std::vector<int> ie_verts;  // 4 per: uv vertices [side][0..1]
    // SELL-32 pattern over rows sorted by length within windows of `sigma` rows
    int n_slices = 0, n_tpanels = 0, sigma = 32;
    std::vector<int> slice_rows, slice_width, slice_tpanel0;
    std::vector<int> rowmap;    // n_slices * 32: local row of (slice, lane)
    std::vector<int> row2slot;  // n_nodes: slice * 32 + lane of each local row
    std::vector<int> tcol;                 // n_tpanels * 32 (local node ids)
    std::vector<int> tcptr;                // n_tpanels * 32 + 1
    std::vector<uint32_t> tcontrib;
    // block-CSR view for cs_get_system: per row, columns sorted, and the SELL slot of each
    std::vector<int> csr_ptr, csr_col, csr_slot;
    long long nnzb = 0;
    // one-ring mesh neighbours (nodes sharing a face edge), sorted, for the learned warm start
    std::vector<int> nbr_ptr, nbr;
    // every edge (reference order): nodes, adjacent faces per side (-1: none); per face its
    // edges (v0 v1), (v1 v2), (v2 v0); per node its (face, corner) pairs in face order
    std::vector<int> e_nodes, e_faces, f_edges, nf_ptr, nf_code;
    // assembly row lists: per node its (face << 2 | corner) in face order and its (interior
    // edge << 2 | corner) in edge order, each with the slots (positions in the node's row) of
    // the element's corners, 8 bits per corner
    std::vector<int> rf_ptr, re_ptr;
    std::vector<int2> rf, re;
    // rest (uv) coordinates of every node, from the first sheet of this connectivity: the
    // geometry the coarse-space segments of the cluster-resident solver are cut along
    std::vector<float> node_uv;
};

struct TopoKey {
    int nn, nv, nf;
    uint64_t h;
    bool operator<(const TopoKey& o) const {
        if (nn != o.nn) return nn < o.nn;
        if (nv != o.nv) return nv < o.nv;
        if (nf != o.nf) return nf < o.nf;
        return h < o.h;
    }
};

uint64_t hashInts(const int32_t* a, size_t n, uint64_t h) {
    for (size_t i = 0; i < n; i++) {
        h ^= (uint64_t)(uint32_t)a[i] + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    }
    return h;
}

std::shared_ptr<Topo> buildTopo(const cs_sheet_desc& s, std::string& err) {
    auto t = std::make_shared<Topo>();
    const int nn = s.n_nodes, nv = s.n_verts, nf = s.n_faces;
    t->n_nodes = nn;
    t->n_verts = nv;
    t->n_faces = nf;
    t->fx.assign(s.face_nodes, s.face_nodes + 3 * nf);
    t->fu.assign(s.face_verts, s.face_verts + 3 * nf);
    for (int i = 0; i < 3 * nf; i++) {
        if (t->fx[i] < 0 || t->fx[i] >= nn || t->fu[i] < 0 || t->fu[i] >= nv) {
            err = "face index out of range";
            return nullptr;
        }
    }
    t->node_uv.assign(2 * (size_t)nn, 0.0f);
    {
        std::vector<char> seen(nn, 0);
        for (int i = 0; i < 3 * nf; i++)
            if (!seen[t->fx[i]]) {
                seen[t->fx[i]] = 1;
                t->node_uv[2 * t->fx[i]] = s.uv[2 * t->fu[i]];
                t->node_uv[2 * t->fx[i] + 1] = s.uv[2 * t->fu[i] + 1];
            }
    }
    // Edges: first appearance order, nodes[0] < nodes[1]; sides per Edge::initialize.
    std::unordered_map<uint64_t, int> map;
    map.reserve(3 * (size_t)nf);
    std::vector<int> eN, eF, eV, eO;
    auto find = [&](int a, int b) {
        if (a > b) std::swap(a, b);
        uint64_t key = (uint64_t)(uint32_t)a << 32 | (uint32_t)b;
        auto it = map.find(key);
        if (it != map.end()) return it->second;
        int id = (int)eN.size() / 2;
        map.emplace(key, id);
        eN.push_back(a); eN.push_back(b);
        eF.push_back(-1); eF.push_back(-1);
        for (int i = 0; i < 4; i++) eV.push_back(-1);
        eO.push_back(-1); eO.push_back(-1);
        return id;
    };
    auto init = [&](int e, int oppCorner, int f) {
        for (int i = 0; i < 3; i++) {
            int c0 = i, c1 = (i + 1) % 3;
            int n0 = t->fx[3 * f + c0], n1 = t->fx[3 * f + c1];
            if (eN[2 * e] == n0 && eN[2 * e + 1] == n1) {
                eV[4 * e] = t->fu[3 * f + c0];
                eV[4 * e + 1] = t->fu[3 * f + c1];
                eO[2 * e] = 3 * f + oppCorner;
                eF[2 * e] = f;
                return;
            } else if (eN[2 * e + 1] == n0 && eN[2 * e] == n1) {
                eV[4 * e + 2] = t->fu[3 * f + c1];
                eV[4 * e + 3] = t->fu[3 * f + c0];
                eO[2 * e + 1] = 3 * f + oppCorner;
                eF[2 * e + 1] = f;
                return;
            }
        }
    };
    for (int f = 0; f < nf; f++) {
        int a = t->fx[3 * f], b = t->fx[3 * f + 1], c = t->fx[3 * f + 2];
        if (a == b || b == c || a == c) {
            err = "degenerate face (repeated node)";
            return nullptr;
        }
        int e0 = find(a, b), e1 = find(b, c), e2 = find(c, a);
        init(e0, 2, f);
        init(e1, 0, f);
        init(e2, 1, f);
        t->f_edges.insert(t->f_edges.end(), {e0, e1, e2});
    }
    const int ne = (int)eN.size() / 2;
    t->e_nodes = eN;
    t->e_faces = eF;
    t->nf_ptr.assign(nn + 1, 0);
    for (int i = 0; i < 3 * nf; i++) t->nf_ptr[t->fx[i] + 1]++;
    for (int i = 0; i < nn; i++) t->nf_ptr[i + 1] += t->nf_ptr[i];
    t->nf_code.resize(3 * (size_t)nf);
    {
        std::vector<int> fill(t->nf_ptr.begin(), t->nf_ptr.end() - 1);
        for (int f = 0; f < nf; f++)
            for (int k = 0; k < 3; k++) t->nf_code[fill[t->fx[3 * f + k]]++] = (f << 2) | k;
    }
    for (int e = 0; e < ne; e++) {
        if (eF[2 * e] < 0 || eF[2 * e + 1] < 0) continue;
        int n0 = eN[2 * e], n1 = eN[2 * e + 1];
        int o0 = t->fx[eO[2 * e]], o1 = t->fx[eO[2 * e + 1]];
        int f0 = eF[2 * e], f1 = eF[2 * e + 1];
        // rotation r with fx[f][0] = (n0, n1, o0)[r] for face 0 and (n1, n0, o1)[r] for face 1
        int ta[3] = {n0, n1, o0}, tb[3] = {n1, n0, o1};
        int r0 = -1, r1 = -1;
        for (int r = 0; r < 3; r++) {
            if (ta[r] == t->fx[3 * f0] && ta[(r + 1) % 3] == t->fx[3 * f0 + 1]) r0 = r;
            if (tb[r] == t->fx[3 * f1] && tb[(r + 1) % 3] == t->fx[3 * f1 + 1]) r1 = r;
        }
        if (r0 < 0 || r1 < 0) {
            err = "inconsistent face orientation";
            return nullptr;
        }
        t->ie_nodes.insert(t->ie_nodes.end(), {n0, n1, o0, o1});
        t->ie_faces.insert(t->ie_faces.end(), {f0, f1});
        t->ie_meta.push_back(r0 | (r1 << 2));
        t->ie_verts.insert(t->ie_verts.end(), {eV[4 * e], eV[4 * e + 1], eV[4 * e + 2], eV[4 * e + 3]});
    }
    const int nie = (int)t->ie_meta.size();
    if (nie >= (1 << 27) || nf >= (1 << 27)) {
        err = "sheet too large for the contributor encoding";
        return nullptr;
    }

    // Contributions per row in the reference's order: faces by index, then interior edges.
    std::vector<int> cnt(nn + 1, 0);
    for (int f = 0; f < nf; f++)
        for (int a = 0; a < 3; a++) cnt[t->fx[3 * f + a] + 1] += 3;
    for (int e = 0; e < nie; e++)
        for (int a = 0; a < 4; a++) cnt[t->ie_nodes[4 * e + a] + 1] += 4;
    for (int i = 0; i < nn; i++) cnt[i + 1] += cnt[i];
    std::vector<uint64_t> rc(cnt[nn]);  // (col << 32) | code, per row, stable-sorted by col
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int f = 0; f < nf; f++)
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                int i = t->fx[3 * f + a], j = t->fx[3 * f + b];
                rc[fill[i]++] = ((uint64_t)(uint32_t)j << 32) | cs_code(0, f, a, b);
            }
    for (int e = 0; e < nie; e++)
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                int i = t->ie_nodes[4 * e + a], j = t->ie_nodes[4 * e + b];
                rc[fill[i]++] = ((uint64_t)(uint32_t)j << 32) | cs_code(1, e, a, b);
            }
    // per row: columns (diagonal first, then ascending) and contributor ranges
    std::vector<std::vector<int>> rowCols(nn);
    std::vector<std::vector<std::pair<int, int>>> rowRanges(nn);
    for (int i = 0; i < nn; i++) {
        auto beg = rc.begin() + cnt[i], end = rc.begin() + cnt[i + 1];
        std::stable_sort(beg, end, [](uint64_t a, uint64_t b) { return (a >> 32) < (b >> 32); });
        std::vector<int> cols;
        std::vector<std::pair<int, int>> ranges;
        cols.push_back(i);
        ranges.push_back({0, 0});
        for (int p = cnt[i]; p < cnt[i + 1];) {
            int j = (int)(rc[p] >> 32);
            int q = p;
            while (q < cnt[i + 1] && (int)(rc[q] >> 32) == j) q++;
            if (j == i)
                ranges[0] = {p, q};
            else {
                cols.push_back(j);
                ranges.push_back({p, q});
            }
            p = q;
        }
        rowCols[i] = std::move(cols);
        rowRanges[i] = std::move(ranges);
    }
    // SELL-32 slices.  Rows are sorted by block count (descending, stable) within windows of
    // sigma rows; sigma is chosen from {32, 64, 128, 256} to minimise the padded slots (the
    // SpMV reads every slot of a slice's width), the smaller window on ties to keep locality.
    std::vector<int> len(nn);
    for (int i = 0; i < nn; i++) len[i] = (int)rowCols[i].size();
    auto orderFor = [&](int sigma) {
        std::vector<int> order(nn);
        for (int i = 0; i < nn; i++) order[i] = i;
        if (sigma > CS_SLICE)
            for (int w0 = 0; w0 < nn; w0 += sigma) {
                int w1 = std::min(nn, w0 + sigma);
                std::stable_sort(order.begin() + w0, order.begin() + w1, [&](int a, int b) { return len[a] > len[b]; });
            }
        return order;
    };
    auto padded = [&](const std::vector<int>& order) {
        long long tot = 0;
        for (int r0 = 0; r0 < nn; r0 += CS_SLICE) {
            int r1 = std::min(nn, r0 + CS_SLICE), w = 1;
            for (int r = r0; r < r1; r++) w = std::max(w, len[order[r]]);
            tot += (long long)w * (r1 - r0);
        }
        return tot;
    };
    std::vector<int> order = orderFor(CS_SLICE);
    long long best = padded(order);
    t->sigma = CS_SLICE;
    for (int sigma : {64, 128, 256}) {
        std::vector<int> o = orderFor(sigma);
        long long p = padded(o);
        if (p < best) {
            best = p;
            order = o;
            t->sigma = sigma;
        }
    }
    t->n_slices = (nn + CS_SLICE - 1) / CS_SLICE;
    t->rowmap.assign((size_t)t->n_slices * CS_SLICE, 0);
    t->row2slot.assign(nn, 0);
    for (int r = 0; r < nn; r++) {
        t->rowmap[r] = order[r];
        t->row2slot[order[r]] = r;
    }
    int tp = 0;
    for (int s = 0; s < t->n_slices; s++) {
        int r0 = s * CS_SLICE, rows = std::min(CS_SLICE, nn - r0);
        int w = 1;
        for (int l = 0; l < rows; l++) w = std::max(w, (int)rowCols[order[r0 + l]].size());
        t->slice_rows.push_back(rows);
        t->slice_width.push_back(w);
        t->slice_tpanel0.push_back(tp);
        tp += w;
    }
    t->n_tpanels = tp;
    t->tcol.assign((size_t)tp * CS_SLICE, 0);
    t->tcptr.assign((size_t)tp * CS_SLICE + 1, 0);
    t->tcontrib.clear();
    t->tcontrib.reserve(rc.size());
    std::vector<int> slotOf;  // per (row, column position)
    std::vector<int> rowSlotBase(nn + 1, 0);
    for (int i = 0; i < nn; i++) rowSlotBase[i + 1] = rowSlotBase[i] + (int)rowCols[i].size();
    slotOf.assign(rowSlotBase[nn], -1);
    for (int s = 0; s < t->n_slices; s++) {
        int r0 = s * CS_SLICE;
        for (int k = 0; k < t->slice_width[s]; k++)
            for (int l = 0; l < CS_SLICE; l++) {
                size_t slot = (size_t)(t->slice_tpanel0[s] + k) * CS_SLICE + l;
                t->tcptr[slot] = (int)t->tcontrib.size();
                if (l < t->slice_rows[s]) {
                    int i = order[r0 + l];
                    if (k < (int)rowCols[i].size()) {
                        t->tcol[slot] = rowCols[i][k];
                        auto rg = rowRanges[i][k];
                        for (int p = rg.first; p < rg.second; p++) t->tcontrib.push_back((uint32_t)(rc[p] & 0xffffffffu));
                        slotOf[rowSlotBase[i] + k] = (int)slot;
                    } else {
                        t->tcol[slot] = i;  // padding: zero block on the diagonal column
                    }
                }
            }
    }
    t->tcptr[(size_t)tp * CS_SLICE] = (int)t->tcontrib.size();
    // Row lists of the assembly gather.  Walking a row's faces, then its edges, in index order
    // and adding each element's blocks onto the slots of its corners visits every block's
    // contributors in the order of the lists above (faces by index, then edges, per element
    // by corner).
    {
        auto slotIn = [&](int i, int j) {
            const auto& cols = rowCols[i];
            for (size_t k = 0; k < cols.size(); k++)
                if (cols[k] == j) return (int)k;
            return -1;
        };
        for (int i = 0; i < nn; i++)
            if (rowCols[i].size() > 255) {
                err = "a node couples to more than 255 nodes";
                return nullptr;
            }
        t->rf_ptr.assign(nn + 1, 0);
        t->rf.resize(3 * (size_t)nf);
        for (int i = 0; i < nn; i++) {
            t->rf_ptr[i + 1] = t->nf_ptr[i + 1];
            for (int q = t->nf_ptr[i]; q < t->nf_ptr[i + 1]; q++) {
                const int f = t->nf_code[q] >> 2;
                int slots = 0;
                for (int b = 0; b < 3; b++) slots |= slotIn(i, t->fx[3 * f + b]) << (8 * b);
                t->rf[q] = make_int2(t->nf_code[q], slots);
            }
        }
        std::vector<int> cntE(nn + 1, 0);
        for (int e = 0; e < nie; e++)
            for (int a = 0; a < 4; a++) cntE[t->ie_nodes[4 * e + a] + 1]++;
        for (int i = 0; i < nn; i++) cntE[i + 1] += cntE[i];
        t->re_ptr = cntE;
        t->re.resize(4 * (size_t)nie);
        std::vector<int> fillE(cntE.begin(), cntE.end() - 1);
        for (int e = 0; e < nie; e++)
            for (int a = 0; a < 4; a++) {
                const int i = t->ie_nodes[4 * e + a];
                int slots = 0;
                for (int b = 0; b < 4; b++) slots |= slotIn(i, t->ie_nodes[4 * e + b]) << (8 * b);
                t->re[fillE[i]++] = make_int2((e << 2) | a, slots);
            }
    }
    // block-CSR view
    t->csr_ptr.assign(nn + 1, 0);
    t->csr_col.clear();
    t->csr_slot.clear();
    for (int i = 0; i < nn; i++) {
        std::vector<std::pair<int, int>> cs;
        for (size_t k = 0; k < rowCols[i].size(); k++) cs.push_back({rowCols[i][k], slotOf[rowSlotBase[i] + k]});
        std::sort(cs.begin(), cs.end());
        for (auto& c : cs) {
            t->csr_col.push_back(c.first);
            t->csr_slot.push_back(c.second);
        }
        t->csr_ptr[i + 1] = (int)t->csr_col.size();
    }
    t->nnzb = (long long)t->csr_col.size();
    // one-ring neighbours
    {
        std::vector<std::vector<int>> nb(nn);
        for (int f = 0; f < nf; f++)
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    if (a != b) nb[t->fx[3 * f + a]].push_back(t->fx[3 * f + b]);
        t->nbr_ptr.assign(nn + 1, 0);
        for (int i = 0; i < nn; i++) {
            std::sort(nb[i].begin(), nb[i].end());
            nb[i].erase(std::unique(nb[i].begin(), nb[i].end()), nb[i].end());
            t->nbr_ptr[i + 1] = t->nbr_ptr[i] + (int)nb[i].size();
            t->nbr.insert(t->nbr.end(), nb[i].begin(), nb[i].end());
        }
    }
    return t;
}

// Cluster-resident solve plan for one topology: contiguous slice ranges per CTA rank with
// balanced panel counts.  Returns the largest number of slices a rank gets.
int residentSplit(const Topo& T, int ncta, std::vector<int>& split) {
    split.assign(CS_RES_MAX_CL + 1, T.n_slices);
    std::vector<long long> pre(T.n_slices + 1, 0);
    for (int i = 0; i < T.n_slices; i++) pre[i + 1] = pre[i] + T.slice_width[i];
    split[0] = 0;
    for (int c = 1; c < ncta; c++) {
        const double target = (double)pre[T.n_slices] * c / ncta;
        int sl = (int)(std::lower_bound(pre.begin(), pre.end(), (long long)std::ceil(target)) - pre.begin());
        if (sl > 0 && target - pre[sl - 1] < pre[sl] - target) sl--;
        split[c] = std::max(split[c - 1], std::min(sl, T.n_slices));
    }
    int w = 0;
    for (int c = 0; c < ncta; c++) w = std::max(w, split[c + 1] - split[c]);
    return w;
}

// Halo plan of one topology on a cluster of `ncta` CTAs.  CTA c owns the rows of slices
// [split[c], split[c+1]) at local slots (slice - split[c]) * 32 + lane.  Every column a CTA's
// rows reference that another CTA owns gets a halo slot in the reading CTA, numbered by
// (owner rank, owner slot).  code: per panel slot, the local p index of its column (own slot,
// or CS_RES_HALO_BIT | halo index, rebased once the batch's own-slot count is known).  send:
// per owner CTA (sendptr), the entries src slot | dst rank << 12 | dst halo index << 16.
struct CoarsePlan {
    int K = 0, nc = 0;             // segments per strip, coarse unknowns (3 per aggregate)
    std::vector<int> agg;          // per local row: rank * K + segment
    std::vector<int> wmask;        // CS_RES_MAX_CL x CS_RES_MAX_WARPS: segments among each warp's rows (bits)
    std::vector<int4> pairs;       // coarse block pairs {a, b, first, last contributor}
    std::vector<int> contrib;      // topology slots of the stored blocks, per pair ascending
};

struct ResidentPlan {
    std::vector<int> split, code, sendptr, halo_count;
    std::vector<uint32_t> send;
    int w = 0, max_halo = 0, max_panels = 0, max_width = 0;
    long long blocks = 0, local_blocks = 0;  // pattern blocks; those with row and column on one CTA
    CoarsePlan coarse;
};

// Segments per strip of the coarse-space correction on a cluster of `ncta` CTAs; CS_COARSE_SEGMENTS
// (0..CS_COARSE_MAX_K, at most CS_COARSE_AGGS / ncta) sets it, 0 turns the correction off.
int coarseSegments(int ncta) {
    const int cap = CS_COARSE_AGGS / std::max(ncta, 1);
    if (const char* ev = std::getenv("CS_COARSE_SEGMENTS")) return std::max(0, std::min({std::atoi(ev), CS_COARSE_MAX_K, cap}));
    return std::min(CS_COARSE_MAX_K, cap);
}

// Shared memory of the coarse region of the resident kernel (resident.cu lays it out the same
// way, each part rounded up to 4 floats): the CTA's rows of the inverse coarse matrix (3K x nc
// floats), the coarse residual in FP32 (nc), the
// correction of the CTA's aggregates and its partial sums (CP = 3K rounded up to 4, each), the
// partials of every CTA in two buffers (2 x ncta x CP), then the coarse residual and search
// direction in FP64 (nc each).
size_t coarseSmemBytes(int ncta, int K) {
    if (K <= 0) return 0;
    auto r4 = [](size_t n) { return (n + 3) / 4 * 4; };  // every part starts on 16 bytes
    const size_t nc = 3 * (size_t)ncta * K, cp = r4(3 * (size_t)K);
    const size_t f = r4(3 * (size_t)K * nc) + r4(nc) + 2 * cp + 2 * (size_t)ncta * cp;
    return f * sizeof(float) + 2 * nc * sizeof(double);
}

// Reorders the lanes of every SELL slice of a topology so that rows of one coarse aggregate sit
// in consecutive lanes (stable within an aggregate).  A slice keeps its rows and width; only
// which lane holds which row changes, with every slot-indexed array (columns, contributor
// lists, the block-CSR view's slots) moved along.  Per warp, the resident solver then sums a
// vector over each aggregate with one segmented scan.
void permuteLanesByAggregate(Topo& T, const std::vector<int>& agg) {
    const size_t nslot = (size_t)T.n_tpanels * CS_SLICE;
    std::vector<int> newOf(nslot), rowmap = T.rowmap;
    for (int s = 0; s < T.n_slices; s++) {
        const int rows = T.slice_rows[s];
        std::vector<int> perm(rows), lnew(CS_SLICE);
        for (int l = 0; l < rows; l++) perm[l] = l;
        std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
            return agg[T.rowmap[s * CS_SLICE + a]] < agg[T.rowmap[s * CS_SLICE + b]];
        });
        for (int l = 0; l < CS_SLICE; l++) lnew[l] = l;
        for (int pos = 0; pos < rows; pos++) {
            lnew[perm[pos]] = pos;
            rowmap[s * CS_SLICE + pos] = T.rowmap[s * CS_SLICE + perm[pos]];
        }
        for (int k = 0; k < T.slice_width[s]; k++)
            for (int l = 0; l < CS_SLICE; l++)
                newOf[(size_t)(T.slice_tpanel0[s] + k) * CS_SLICE + l] = (T.slice_tpanel0[s] + k) * CS_SLICE + lnew[l];
    }
    std::vector<int> oldOf(nslot), tcol(nslot), tcptr(nslot + 1);
    for (size_t o = 0; o < nslot; o++) oldOf[newOf[o]] = (int)o;
    std::vector<uint32_t> tcontrib;
    tcontrib.reserve(T.tcontrib.size());
    for (size_t q = 0; q < nslot; q++) {
        const int o = oldOf[q];
        tcol[q] = T.tcol[o];
        tcptr[q] = (int)tcontrib.size();
        tcontrib.insert(tcontrib.end(), T.tcontrib.begin() + T.tcptr[o], T.tcontrib.begin() + T.tcptr[o + 1]);
    }
    tcptr[nslot] = (int)tcontrib.size();
    for (int& q : T.csr_slot) q = newOf[q];
    T.rowmap = rowmap;
    for (int s = 0; s < T.n_slices; s++)
        for (int l = 0; l < T.slice_rows[s]; l++) T.row2slot[rowmap[s * CS_SLICE + l]] = s * CS_SLICE + l;
    T.tcol.swap(tcol);
    T.tcptr.swap(tcptr);
    T.tcontrib.swap(tcontrib);
}

// Coarse space of the batched loop for one topology (coarse.cu): the nodes binned by their rest
// (u, v) into g x g cells of the bounding box (g = round(sqrt(nodes / CS_BC_NODES_PER_AGG)),
// 1..gmax), the non-empty cells numbered in cell order as aggregates; members of each
// aggregate ascending; per pair of aggregates, the stored blocks coupling them in slot order.
struct BCPlan {
    int na = 0;
    std::vector<int> agg, mptr, mem, contrib;
    std::vector<int4> pairs;
};

void batchedCoarsePlan(const Topo& T, int gmax, BCPlan& P) {
    P = BCPlan();
    const int n = T.n_nodes;
    if (n <= 0 || (int)T.node_uv.size() < 2 * n) return;
    int g = (int)std::lround(std::sqrt((double)n / CS_BC_NODES_PER_AGG));
    g = std::max(1, std::min(g, gmax));
    float u0 = T.node_uv[0], u1 = u0, v0 = T.node_uv[1], v1 = v0;
    for (int i = 0; i < n; i++) {
        u0 = std::min(u0, T.node_uv[2 * i]);
        u1 = std::max(u1, T.node_uv[2 * i]);
        v0 = std::min(v0, T.node_uv[2 * i + 1]);
        v1 = std::max(v1, T.node_uv[2 * i + 1]);
    }
    const double du = u1 > u0 ? (double)(u1 - u0) : 1.0, dv = v1 > v0 ? (double)(v1 - v0) : 1.0;
    std::vector<int> cell(n), id(g * g, -1);
    for (int i = 0; i < n; i++) {
        const int cu = std::min(g - 1, std::max(0, (int)((T.node_uv[2 * i] - u0) / du * g)));
        const int cv = std::min(g - 1, std::max(0, (int)((T.node_uv[2 * i + 1] - v0) / dv * g)));
        cell[i] = cu * g + cv;
        id[cell[i]] = 0;
    }
    for (int k = 0; k < g * g; k++)
        if (id[k] == 0) id[k] = P.na++;
    P.agg.resize(n);
    P.mptr.assign(P.na + 1, 0);
    for (int i = 0; i < n; i++) {
        P.agg[i] = id[cell[i]];
        P.mptr[P.agg[i] + 1]++;
    }
    for (int a = 0; a < P.na; a++) P.mptr[a + 1] += P.mptr[a];
    P.mem.resize(n);
    std::vector<int> fill(P.mptr.begin(), P.mptr.end() - 1);
    for (int i = 0; i < n; i++) P.mem[fill[P.agg[i]]++] = i;
    // coarse pattern: every stored block (slots with contributors; padding has none)
    std::vector<std::tuple<int, int, int>> blk;
    for (int sl = 0; sl < T.n_slices; sl++)
        for (int k = 0; k < T.slice_width[sl]; k++)
            for (int l = 0; l < T.slice_rows[sl]; l++) {
                const int slot = (T.slice_tpanel0[sl] + k) * CS_SLICE + l;
                if (T.tcptr[slot + 1] == T.tcptr[slot]) continue;
                blk.emplace_back(P.agg[T.rowmap[sl * CS_SLICE + l]], P.agg[T.tcol[slot]], slot);
            }
    std::sort(blk.begin(), blk.end());
    for (size_t i = 0; i < blk.size();) {
        size_t j = i;
        while (j < blk.size() && std::get<0>(blk[j]) == std::get<0>(blk[i]) && std::get<1>(blk[j]) == std::get<1>(blk[i])) j++;
        P.pairs.push_back(make_int4(std::get<0>(blk[i]), std::get<1>(blk[i]), (int)P.contrib.size(),
                                    (int)(P.contrib.size() + (j - i))));
        for (size_t q = i; q < j; q++) P.contrib.push_back(std::get<2>(blk[q]));
        i = j;
    }
}

// Coarse-space plan of one topology on a cluster of `ncta` CTAs: each CTA's strip of rows is cut
// into K segments of equal row count along the principal axis of the rows' rest coordinates (a
// strip of a grid sheet is a band of grid rows; its segments are blocks side by side), and the
// coarse pattern lists, per pair of aggregates, the stored blocks coupling them in slot order.
void coarsePlan(const Topo& T, ResidentPlan& P, int ncta, int K) {
    CoarsePlan& C = P.coarse;
    C = CoarsePlan();
    C.K = K;
    C.nc = 3 * ncta * K;
    C.agg.assign(T.n_nodes, -1);
    C.wmask.assign(CS_RES_MAX_CL * CS_RES_MAX_WARPS, 0);
    for (int c = 0; c < ncta; c++) {
        std::vector<std::pair<int, int>> rows;  // (local row, own slot)
        for (int sl = P.split[c]; sl < P.split[c + 1]; sl++)
            for (int l = 0; l < T.slice_rows[sl]; l++)
                rows.push_back({T.rowmap[sl * CS_SLICE + l], (sl - P.split[c]) * CS_SLICE + l});
        const int n = (int)rows.size();
        double mx = 0.0, my = 0.0;
        for (auto& r : rows) {
            mx += T.node_uv[2 * r.first];
            my += T.node_uv[2 * r.first + 1];
        }
        mx /= std::max(n, 1);
        my /= std::max(n, 1);
        double sxx = 0.0, sxy = 0.0, syy = 0.0;
        for (auto& r : rows) {
            const double dx = T.node_uv[2 * r.first] - mx, dy = T.node_uv[2 * r.first + 1] - my;
            sxx += dx * dx;
            sxy += dx * dy;
            syy += dy * dy;
        }
        // principal axis: eigenvector of the larger eigenvalue of the 2x2 scatter matrix
        const double tr = sxx + syy, det = sxx * syy - sxy * sxy;
        const double l1 = 0.5 * tr + std::sqrt(std::max(0.0, 0.25 * tr * tr - det));
        double ax = 1.0, ay = 0.0;
        if (std::fabs(sxy) > 0.0) {
            ax = l1 - syy;
            ay = sxy;
        } else if (syy > sxx) {
            ax = 0.0;
            ay = 1.0;
        }
        std::vector<std::pair<double, int>> key(n);
        for (int i = 0; i < n; i++) {
            const int r = rows[i].first;
            key[i] = {(T.node_uv[2 * r] - mx) * ax + (T.node_uv[2 * r + 1] - my) * ay, i};
        }
        std::sort(key.begin(), key.end());
        for (int k = 0; k < K; k++)
            for (int i = (int)((long long)k * n / K); i < (int)((long long)(k + 1) * n / K); i++) {
                const auto& r = rows[key[i].second];
                C.agg[r.first] = c * K + k;
                C.wmask[c * CS_RES_MAX_WARPS + r.second / CS_SLICE] |= 1 << k;  // own slot / 32 = warp
            }
    }
    // coarse pattern: every stored block (slots with contributors; padding has none)
    std::vector<std::tuple<int, int, int>> blk;  // (a, b, slot)
    for (int sl = 0; sl < T.n_slices; sl++)
        for (int k = 0; k < T.slice_width[sl]; k++)
            for (int l = 0; l < T.slice_rows[sl]; l++) {
                const int slot = (T.slice_tpanel0[sl] + k) * CS_SLICE + l;
                if (T.tcptr[slot + 1] == T.tcptr[slot]) continue;
                blk.emplace_back(C.agg[T.rowmap[sl * CS_SLICE + l]], C.agg[T.tcol[slot]], slot);
            }
    std::sort(blk.begin(), blk.end());
    for (size_t i = 0; i < blk.size();) {
        size_t j = i;
        while (j < blk.size() && std::get<0>(blk[j]) == std::get<0>(blk[i]) && std::get<1>(blk[j]) == std::get<1>(blk[i])) j++;
        C.pairs.push_back(make_int4(std::get<0>(blk[i]), std::get<1>(blk[i]), (int)C.contrib.size(),
                                    (int)(C.contrib.size() + (j - i))));
        for (size_t q = i; q < j; q++) C.contrib.push_back(std::get<2>(blk[q]));
        i = j;
    }
}

#define CS_RES_HALO_BIT 0x40000000

ResidentPlan residentPlan(const Topo& T, int ncta) {
    ResidentPlan P;
    P.w = residentSplit(T, ncta, P.split);
    const int nn = T.n_nodes;
    std::vector<int> owner(nn, 0), oslot(nn, 0);
    for (int c = 0; c < ncta; c++)
        for (int sl = P.split[c]; sl < P.split[c + 1]; sl++)
            for (int l = 0; l < T.slice_rows[sl]; l++) {
                owner[T.rowmap[sl * CS_SLICE + l]] = c;
                oslot[T.rowmap[sl * CS_SLICE + l]] = (sl - P.split[c]) * CS_SLICE + l;
            }
    P.code.assign(T.tcol.size(), 0);
    P.halo_count.assign(CS_RES_MAX_CL + 1, 0);
    std::vector<std::vector<std::pair<int, int>>> halo(ncta);  // per reader: (owner, owner slot) sorted
    for (int c = 0; c < ncta; c++) {
        std::vector<std::pair<int, int>> need;
        int np = 0;
        for (int sl = P.split[c]; sl < P.split[c + 1]; sl++) {
            np += T.slice_width[sl];
            P.max_width = std::max(P.max_width, T.slice_width[sl]);
            for (int k = 0; k < T.slice_width[sl]; k++)
                for (int l = 0; l < T.slice_rows[sl]; l++) {
                    const int col = T.tcol[(size_t)(T.slice_tpanel0[sl] + k) * CS_SLICE + l];
                    if (owner[col] != c) need.push_back({owner[col], oslot[col]});
                }
        }
        P.max_panels = std::max(P.max_panels, np);
        std::sort(need.begin(), need.end());
        need.erase(std::unique(need.begin(), need.end()), need.end());
        halo[c] = need;
        P.max_halo = std::max(P.max_halo, (int)need.size());
        P.halo_count[c] = (int)need.size();
        for (int sl = P.split[c]; sl < P.split[c + 1]; sl++)
            for (int k = 0; k < T.slice_width[sl]; k++)
                for (int l = 0; l < T.slice_rows[sl]; l++) {
                    const size_t slot = (size_t)(T.slice_tpanel0[sl] + k) * CS_SLICE + l;
                    const int col = T.tcol[slot];
                    if (owner[col] == c) {
                        P.code[slot] = oslot[col];
                    } else {
                        auto it = std::lower_bound(need.begin(), need.end(), std::make_pair(owner[col], oslot[col]));
                        P.code[slot] = CS_RES_HALO_BIT | (int)(it - need.begin());
                    }
                }
    }
    for (int i = 0; i < nn; i++)
        for (int q = T.csr_ptr[i]; q < T.csr_ptr[i + 1]; q++) {
            P.blocks++;
            P.local_blocks += owner[T.csr_col[q]] == owner[i];
        }
    P.sendptr.assign(CS_RES_MAX_CL + 1, 0);
    for (int c = 0; c < ncta; c++) {
        P.sendptr[c] = (int)P.send.size();
        for (int d = 0; d < ncta; d++)
            for (size_t h = 0; h < halo[d].size(); h++)
                if (halo[d][h].first == c)
                    P.send.push_back((uint32_t)halo[d][h].second | ((uint32_t)d << 12) | ((uint32_t)h << 16));
    }
    for (int c = ncta; c <= CS_RES_MAX_CL; c++) P.sendptr[c] = (int)P.send.size();
    return P;
}

}  // namespace

// ---------------------------------------------------------------------------------------

// Device buffers of the proximity terms, grown as needed (applyProximities).
struct ProxBuffers {
    cs_proximity_desc* desc = nullptr;  // the proximities in force
    int* icount = nullptr;              // instances per proximity, then their offsets
    ProxInst* inst = nullptr;
    float* rec = nullptr;
    int* rowPtr = nullptr;              // N + 1
    int* rowFill = nullptr;             // N + 1
    int* xptr = nullptr;                // N + 1
    int* rowInst = nullptr;
    int* xcol = nullptr;
    float* xval = nullptr;
    int* sheetProx = nullptr;
    int* partial = nullptr;             // scan block sums
    size_t descCap = 0, icountCap = 0, instCap = 0, recCap = 0, rowCap = 0, rowFillCap = 0, xptrCap = 0,
           rowInstCap = 0, xcolCap = 0, xvalCap = 0, sheetCap = 0, partialCap = 0;
    int n = 0;  // proximities in force
    void release() {
        void* ps[] = {desc, icount, inst, rec, rowPtr, rowFill, xptr, rowInst, xcol, xval, sheetProx, partial};
        for (void* q : ps)
            if (q) cudaFree(q);
        *this = ProxBuffers();
    }
};

struct CollideCaps {
    size_t found = 0, all = 0;
};

struct cs_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // a second stream for the resident coarse set-up, forked after the assembly and joined before
    // the resident solve (it overlaps the learned inference and the solve set-up)
    cudaStream_t side = nullptr;
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    std::string err;
    Batch B;
    bool loaded = false;
    std::vector<void*> allocs;
    // host copies needed by the inspection entry points
    std::vector<SheetDesc> sheets;
    std::vector<SliceDesc> slices;
    std::vector<std::shared_ptr<Topo>> sheetTopo;
    long long nnzb_pattern = 0;
    // graphs of the step, per [learned warm start][coarse-correction kernels in the loop trips]
    cudaGraphExec_t gexec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    cudaGraph_t gph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    // launchTrip launches the batched coarse correction's kernels (the step asks for it); the
    // launch counter's trips before the last change of this setting and their kernels
    bool tripCoarse = true;
    long long tripsBase = 0, tripLaunchBase = 0;
    DevParams hostParams{};
    bool lastStepValid = false;
    long long steps = 0, hostLaunches = 0, graphSteps = 0, graphLaunchesFixed = 0;
    int gatherGrid = 1;  // persistent assembly gather: a few warps per SM walk the slices
    size_t gatherSmem = 0;  // its dynamic shared memory (slot accumulators)
    int gatherWarps = 1;    // its warps per CTA
    // learned warm start
    MlpDev mlp;
    bool mlpInit = false;
    int mlpGridTile = 0, mlpGridTrain = 0;
    int mlpGridL1 = 0, mlpGridL23 = 0;  // inference grids: resident CTAs per SM (TMEM: 512 columns per SM)
    long long adamStep = 0;
    float* mlpScratch = nullptr;  // per-epoch loss accumulators, gradient output
    // cluster-resident solver launch (resident.cu): CTAs per cluster, threads per CTA,
    // clusters in the persistent grid, dynamic shared memory per CTA
    int resCL = 0, resThreads = 0, resClusters = 0, resClustersMax = 0;
    int spmvShape = CS_SPMV_DEFAULT;    // launch shape of the batched SpMV (cs_tune)
    int tunedDegree = 0, tunedCoarse = 0;  // fastest resident preconditioner found by cs_tune (0: not tuned)
    int tunedSolver = -1;                  // faster solve route found by cs_tune (-1: not tuned)
    size_t bcSmemBig = 0;                  // dynamic shared memory of cs_bc_invert_cluster_kernel
    long long bcMatFloats = 0;             // floats of the batched loop's coarse matrices
    bool energyBegun = false;              // cs_mlp_energy_begin ran; cs_mlp_energy_end not yet
    int energyLoopCap = 0;                 // the begun step's trip bound (its statistics)
    std::vector<int> handleNode;  // batch node of every handle, in load order (cs_set_handle_motions)
    int maxHandleMotion = -1;     // largest motion a handle follows (-1: none)
    size_t resSmem = 0;
    std::vector<int> rlistAll;  // resident sheets before the proximity filter
    std::vector<int> rlistCur;  // resident sheets now
    std::vector<long long> sheetBlocks, sheetLocalBlocks;  // per sheet: pattern blocks, strip-local ones
    // proximities (cs_set_proximities): their device lists, and the host copies of the
    // blocks outside the pattern that cs_get_system merges
    ProxBuffers prox;
    // proximity detection (contact.cu): static scene data built at the first detection
    Contact contact;
    bool contactReady = false;
    int* sheetGroupDev = nullptr;
    std::vector<void*> contactAllocs;
    // collision step (collide.cu)
    Collide coll;
    CollideCaps collCaps;
};

namespace {

cs_status fail(cs_ctx* c, cs_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return st;
}

#define CS_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(c, CS_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <class T>
cs_status dalloc(cs_ctx* c, T** p, size_t count) {
    if (count == 0) count = 1;
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e != cudaSuccess) return fail(c, CS_ERR_CUDA, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
    c->allocs.push_back(q);
    *p = (T*)q;
    return CS_OK;
}

template <class T>
cs_status upload(cs_ctx* c, T** p, const std::vector<T>& h) {
    cs_status st = dalloc(c, p, h.size());
    if (st != CS_OK) return st;
    if (!h.empty()) CS_CUDA(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return CS_OK;
}

void freeBatch(cs_ctx* c) {
    c->spmvShape = CS_SPMV_DEFAULT;
    c->tunedDegree = c->tunedCoarse = 0;
    c->handleNode.clear();
    c->maxHandleMotion = -1;
    for (int l = 0; l < 2; l++)
        for (int k = 0; k < 2; k++) {
            if (c->gexec[l][k]) cudaGraphExecDestroy(c->gexec[l][k]);
            if (c->gph[l][k]) cudaGraphDestroy(c->gph[l][k]);
            c->gexec[l][k] = nullptr;
            c->gph[l][k] = nullptr;
        }
    c->tripCoarse = true;
    c->tripsBase = c->tripLaunchBase = 0;
    c->mlp = MlpDev();
    c->mlpInit = false;
    c->adamStep = 0;
    c->mlpScratch = nullptr;
    for (void* p : c->allocs) cudaFree(p);
    c->allocs.clear();
    c->prox.release();
    for (void* p : c->contactAllocs) cudaFree(p);
    c->contactAllocs.clear();
    if (c->contact.pairs) cudaFree(c->contact.pairs);
    {
        Collide& K = c->coll;
        void* ps[] = {K.found, K.counters, K.sorted, K.all, K.used, K.nodemin, K.alive, K.chosen, K.mark, K.nodes,
                      K.idx, K.nptr, K.nfill, K.nlist, K.x1, K.cur, K.next, K.grad, K.lambda, K.coef,
                      K.cterm, K.nterm, K.gterm, K.skey[0], K.skey[1], K.sperm[0], K.sperm[1], K.stmp};
        for (void* q : ps)
            if (q) cudaFree(q);
        c->coll = Collide();
        c->collCaps = CollideCaps();
    }
    c->contact = Contact();
    c->contactReady = false;
    c->sheetGroupDev = nullptr;
    c->rlistAll.clear();
    c->rlistCur.clear();
    c->B = Batch();
    c->loaded = false;
    c->lastStepValid = false;
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

// Raises a kernel's limit on dynamic shared memory to at least `bytes`, never lowering it.  The
// limit belongs to the function (on the current device), not to a context: every context of
// the process shares it, and batches of different sizes need different amounts, so a context
// loaded later must not take away what an earlier one launches with.
cudaError_t raiseDynSmem(const void* kernel, size_t bytes) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, kernel);
    if (e != cudaSuccess) return e;
    if ((size_t)a.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

int launchAssembly(cs_ctx* c) {
    Batch& B = c->B;
    int n = 1;
    if (B.E) cs_edge_kernel<<<nblk(B.E, 128), 128, 0, c->stream>>>(B), n++;
    cs_gather_kernel<<<c->gatherGrid, 32 * c->gatherWarps, c->gatherSmem, c->stream>>>(B);
    if (B.n_pinst > 0) {
        // proximity terms after the handles (Cloth.cu:676-684): records, then per row the
        // blocks, right-hand side and block-Jacobi inverse, then the ||b|| partials
        cs_prox_kernel<<<nblk(B.n_pinst, 128), 128, 0, c->stream>>>(B);
        cs_prox_row_kernel<<<nblk(B.N, 128), 128, 0, c->stream>>>(B);
        cs_slice_bnorm_kernel<<<nblk((long long)B.n_slices * 32, 128), 128, 0, c->stream>>>(B);
        n += 3;
    }
    return n;
}

// The batched loop's coarse matrices of this step's systems, inverted (coarse.cu; the kernels
// return at once for sheets the loop does not solve or when the step asks for no correction).
int launchBatchedCoarseSetup(cs_ctx* c) {
    Batch& B = c->B;
    if (B.bc_total_agg <= 0) return 0;
    cudaMemsetAsync(B.bc_mat, 0, (size_t)c->bcMatFloats * sizeof(float), c->stream);
    const int gx = std::max(1, std::min(256, nblk(B.bc_max_npair, 8)));
    cs_bc_assemble_kernel<<<dim3(gx, B.S), 256, 0, c->stream>>>(B);
    cs_bc_invert_small_kernel<<<B.S, CS_BC_THREADS, (CS_BC_SMALL_NC * CS_BC_SMALL_NC + 4 + 2 * CS_BC_KB * CS_BC_SMALL_NC + CS_BC_KB * CS_BC_KB) * sizeof(float),
                                c->stream>>>(B);
    int n = 2;
    if (B.bc_n_big > 0) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CS_BC_CLUSTER;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(CS_BC_CLUSTER * B.bc_n_big);
        cfg.blockDim = dim3(CS_BC_THREADS);
        cfg.dynamicSmemBytes = c->bcSmemBig;
        cfg.stream = c->stream;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, cs_bc_invert_cluster_kernel, B);
        n++;
    }
    return n;
}

// Kernels per step of the batched loop's coarse set-up, of the resident solve, and per loop trip
// (the launch counters of cs_get_counters).
// Kernels launchAssembly launches: the edge records, the gather, the proximity terms.
int assemblyKernels(const cs_ctx* c) { return (c->B.E ? 1 : 0) + 1 + (c->B.n_pinst > 0 ? 3 : 0); }
int bcSetupKernels(const cs_ctx* c) { return c->B.bc_total_agg > 0 ? 2 + (c->B.bc_n_big > 0 ? 1 : 0) : 0; }
int residentKernels(const cs_ctx* c) {
    return c->resClusters > 0 ? 1 + (c->B.res_cnc > 0 && c->B.n_resident > 0 ? 1 : 0) : 0;
}
int tripKernels(const cs_ctx* c) { return 4 + (c->B.bc_total_agg > 0 && c->tripCoarse ? 3 : 0); }

// Whether the loop trips launch the batched coarse correction's kernels (only when the step asks
// for the correction: without it they would only return); the launch counter folds the trips
// so far at the old setting.
cs_status setTripCoarse(cs_ctx* c, bool on) {
    if (c->tripCoarse == on) return CS_OK;
    int loopv[8];
    CS_CUDA(cudaMemcpyAsync(loopv, c->B.loop, sizeof(loopv), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    const long long trips = (long long)(unsigned)loopv[4];
    c->tripLaunchBase += (long long)tripKernels(c) * (trips - c->tripsBase);
    c->tripsBase = trips;
    c->tripCoarse = on;
    return CS_OK;
}

void launchSolvePrologue(cs_ctx* c) {
    Batch& B = c->B;
    cs_solve_setup_kernel<<<B.S, 128, 0, c->stream>>>(B);
    launchBatchedCoarseSetup(c);
    cs_solve_prologue_kernel<<<nblk(3LL * B.N, 256), 256, 0, c->stream>>>(B);
}

// A solve set-up for measurements that re-run the solve on an assembled system after other
// kernels have reused the slice partials: the ||b||^2 partials first, as the assembly leaves them.
void launchSolvePrologueAgain(cs_ctx* c) {
    Batch& B = c->B;
    cs_slice_bnorm_kernel<<<nblk((long long)B.n_slices * 32, 128), 128, 0, c->stream>>>(B);
    launchSolvePrologue(c);
}

// Sheets that fit a cluster's shared memory: one persistent cluster per sheet at a time.
// The coarse matrices of the resident sheets, formed and inverted for this step's systems (the
// kernel returns at once unless the step asks for the coarse correction).
void launchCoarseSetup(cs_ctx* c) {
    if (c->resClusters > 0 && c->B.res_cnc > 0 && c->B.n_resident > 0)
        cs_coarse_setup_kernel<<<c->B.n_resident, CS_COARSE_THREADS, cs_coarse_setup_smem(c->B.res_cnc), c->stream>>>(c->B);
}

void launchResident(cs_ctx* c, bool setup = true) {
    if (c->resClusters <= 0) return;
    if (setup) launchCoarseSetup(c);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = c->resCL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(c->resClusters * c->resCL);
    cfg.blockDim = dim3(c->resThreads);
    cfg.dynamicSmemBytes = c->resSmem;
    cfg.stream = c->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, cs_resident_pcg_kernel, c->B);
}

int launchMlpInference(cs_ctx* c, float* pred);

// The step up to its solve loop: assembly; the resident sheets' coarse matrices on the side
// stream while the learned inference (when asked) and the solve set-up run on the main stream;
// the join; the cluster-resident solve.  Captured into the step graph, or launched directly.
void launchPrelude(cs_ctx* c, bool learned) {
    launchAssembly(c);
    const bool fork = c->resClusters > 0 && c->B.res_cnc > 0 && c->B.n_resident > 0;
    if (fork) {
        cudaEventRecord(c->evFork, c->stream);
        cudaStreamWaitEvent(c->side, c->evFork, 0);
        cs_coarse_setup_kernel<<<c->B.n_resident, CS_COARSE_THREADS, cs_coarse_setup_smem(c->B.res_cnc), c->side>>>(c->B);
        cudaEventRecord(c->evJoin, c->side);
    }
    if (learned) launchMlpInference(c, c->B.warm);
    launchSolvePrologue(c);
    if (fork) cudaStreamWaitEvent(c->stream, c->evJoin, 0);
    launchResident(c, false);
}

// Learned warm start: features of the assembled system, layer 1, layers 2-3 + output; the
// prediction replaces the previous dv in B.warm (the solve then starts from it).
int launchMlpInference(cs_ctx* c, float* pred) {
    Batch& B = c->B;
    MlpDev& M = c->mlp;
    cs_mlp_features_kernel<<<nblk(B.N, 256), 256, 0, c->stream>>>(B, M, M.feat);
    cs_mlp_l1_kernel<<<c->mlpGridL1, 128, MLP_SMEM_L1, c->stream>>>(B, M, M.feat, 0, B.N, nullptr);
    cs_mlp_l23_kernel<<<c->mlpGridL23, 128, MLP_SMEM_L23, c->stream>>>(B, M, 0, B.N, nullptr, nullptr, nullptr, pred);
    return 3;
}

void launchTrip(cs_ctx* c, cudaGraphConditionalHandle h) {
    Batch& B = c->B;
    int g = nblk((long long)B.n_slices * 32, 128);
    launchSpmvShape(B, c->spmvShape, c->stream);
    cs_reduce1_kernel<<<B.S, CS_REDUCE_THREADS, 0, c->stream>>>(B);
    cs_vector_kernel<<<g, 128, 0, c->stream>>>(B);
    if (B.bc_total_agg > 0 && c->tripCoarse) {
        // the coarse correction of z and the r.z, r.r partials it changes (coarse.cu)
        cs_bc_restrict_kernel<<<B.bc_total_agg, 256, 0, c->stream>>>(B);
        cs_bc_apply_kernel<<<nblk((long long)B.bc_total_agg * 96, 256), 256, 0, c->stream>>>(B);
        cs_bc_finish_kernel<<<g, 128, 0, c->stream>>>(B);
    }
    cs_reduce2_kernel<<<B.S, CS_REDUCE_THREADS, 0, c->stream>>>(B, h);
}

cs_status buildGraph(cs_ctx* c, bool learned) {
    cudaGraphExec_t& exec = c->gexec[learned][c->tripCoarse];
    if (exec) return CS_OK;
    cudaGraph_t graph;
    CS_CUDA(cudaGraphCreate(&graph, 0));
    c->gph[learned][c->tripCoarse] = graph;
    // prelude: assembly (+ learned warm start) + solve setup, captured into the graph
    CS_CUDA(cudaStreamBeginCaptureToGraph(c->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launchPrelude(c, learned);
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CS_CUDA(cudaStreamGetCaptureInfo(c->stream, &cst, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> prelude(deps, deps + ndeps);
    CS_CUDA(cudaStreamEndCapture(c->stream, &graph));
    // while loop over solve trips
    cudaGraphConditionalHandle handle;
    CS_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loopNode;
    CS_CUDA(cudaGraphAddNode(&loopNode, graph, prelude.data(), prelude.size(), &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CS_CUDA(cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launchTrip(c, handle);
    CS_CUDA(cudaStreamEndCapture(c->stream, &body));
    // epilogue
    CS_CUDA(cudaStreamBeginCaptureToGraph(c->stream, graph, &loopNode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    cs_advance_kernel<<<nblk(3LL * c->B.N, 256), 256, 0, c->stream>>>(c->B);
    CS_CUDA(cudaStreamEndCapture(c->stream, &graph));
    CS_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    return CS_OK;
}

DevParams toDev(const cs_step_params* p) {
    DevParams d{};
    d.dt = p->dt;
    for (int i = 0; i < 3; i++) d.gravity[i] = p->gravity[i];
    d.handle_stiffness = p->handle_stiffness;
    d.tol = p->tol > 0 ? p->tol : 1e-6;
    d.inner_tol = p->inner_tol > 0 ? p->inner_tol : 1e-2;
    d.max_iters = p->max_iters > 0 ? p->max_iters : 2000;
    d.sweep_cap = p->sweep_cap > 0 ? p->sweep_cap : 1000000;
    d.mixed = p->precision == CS_PREC_MIXED;
    d.warm = p->warm_start != CS_WARM_ZERO;
    d.loop_cap = 2 * d.max_iters + 256;
    d.advance = p->advance;
    d.solver = p->solver == CS_SOLVER_BATCHED ? CS_SOLVER_BATCHED_DEV : CS_SOLVER_AUTO_DEV;
    d.warm_scale = p->warm_scale != 0;
    d.cheb_degree = p->precond_degree >= 3 ? p->precond_degree : 1;
    d.coarse = p->coarse != 0;
    d.n_motions = p->transformations ? std::min(std::max(p->n_transformations, 0), CS_MAX_MOTIONS) : 0;
    for (int m = 0; m < d.n_motions; m++)
        for (int k = 0; k < CS_TRANSFORM_FLOATS; k++) d.motion[m][k] = p->transformations[CS_TRANSFORM_FLOATS * m + k];
    return d;
}

}  // namespace

extern "C" {

cs_status cs_create(cs_ctx** out, int device) {
    if (!out) return CS_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return CS_ERR_NO_DEVICE;
    if (device < 0 || device >= n) return CS_ERR_INVALID_ARG;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CS_ERR_NO_DEVICE;
    if (prop.major != 10) return CS_ERR_NO_DEVICE;  // built for sm_100a only
    auto* c = new cs_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evFork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evJoin, cudaEventDisableTiming) != cudaSuccess) {
        delete c;
        return CS_ERR_CUDA;
    }
    *out = c;
    return CS_OK;
}

cs_status cs_destroy(cs_ctx* c) {
    if (!c) return CS_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    freeBatch(c);
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaEventDestroy(c->evFork);
    cudaEventDestroy(c->evJoin);
    cudaStreamDestroy(c->side);
    cudaStreamDestroy(c->stream);
    delete c;
    return CS_OK;
}

const char* cs_last_error(const cs_ctx* c) { return c ? c->err.c_str() : "null context"; }

cs_status cs_load_batch(cs_ctx* c, const cs_material_desc* mats, int n_mats, const cs_sheet_desc* sheets,
                        int n_sheets) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!mats || n_mats <= 0 || !sheets || n_sheets <= 0) return fail(c, CS_ERR_INVALID_ARG, "empty batch");
    CS_CUDA(cudaSetDevice(c->device));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    freeBatch(c);
    // validate
    long long N = 0, F = 0;
    for (int s = 0; s < n_sheets; s++) {
        const cs_sheet_desc& d = sheets[s];
        if (d.n_nodes <= 0 || d.n_faces <= 0 || d.n_verts <= 0 || !d.x || !d.uv || !d.face_nodes || !d.face_verts)
            return fail(c, CS_ERR_INVALID_ARG, "sheet %d: empty or missing arrays", s);
        if (d.material < 0 || d.material >= n_mats) return fail(c, CS_ERR_INVALID_ARG, "sheet %d: bad material", s);
        if (d.n_handles < 0 || (d.n_handles > 0 && !d.handle_nodes))
            return fail(c, CS_ERR_INVALID_ARG, "sheet %d: bad handles", s);
        for (int h = 0; h < d.n_handles; h++)
            if (d.handle_nodes[h] < 0 || d.handle_nodes[h] >= d.n_nodes)
                return fail(c, CS_ERR_INVALID_ARG, "sheet %d: handle node %d out of range", s, d.handle_nodes[h]);
        for (int i = 0; i < 3 * d.n_nodes; i++)
            if (!std::isfinite(d.x[i]) || (d.v && !std::isfinite(d.v[i])))
                return fail(c, CS_ERR_INVALID_ARG, "sheet %d: non-finite node state", s);
        N += d.n_nodes;
        F += d.n_faces;
    }
    if (N >= (1LL << 31) / 9 || F >= (1LL << 31) / 32) return fail(c, CS_ERR_INVALID_ARG, "batch too large");

    // topologies (shared)
    std::map<TopoKey, int> topoIndex;
    std::vector<std::shared_ptr<Topo>> topos;
    c->sheetTopo.assign(n_sheets, nullptr);
    std::vector<int> sheetTopoId(n_sheets);
    for (int s = 0; s < n_sheets; s++) {
        const cs_sheet_desc& d = sheets[s];
        TopoKey k{d.n_nodes, d.n_verts, d.n_faces, 0};
        k.h = hashInts(d.face_nodes, 3 * (size_t)d.n_faces, 1469598103934665603ULL);
        k.h = hashInts(d.face_verts, 3 * (size_t)d.n_faces, k.h);
        auto it = topoIndex.find(k);
        if (it != topoIndex.end() &&
            std::equal(d.face_nodes, d.face_nodes + 3 * d.n_faces, topos[it->second]->fx.begin()) &&
            std::equal(d.face_verts, d.face_verts + 3 * d.n_faces, topos[it->second]->fu.begin())) {
            sheetTopoId[s] = it->second;
        } else {
            std::string err;
            auto t = buildTopo(d, err);
            if (!t) return fail(c, CS_ERR_INVALID_ARG, "sheet %d: %s", s, err.c_str());
            sheetTopoId[s] = (int)topos.size();
            topoIndex[k] = (int)topos.size();
            topos.push_back(t);
        }
        c->sheetTopo[s] = topos[sheetTopoId[s]];
    }
    // materials: scaled stretching tables per distinct (rows, multiplier)
    std::map<std::vector<float>, std::vector<float>> baseSamples;
    std::map<std::vector<float>, int> tableIndex;
    std::vector<float4> tables;
    std::vector<int> sheetTable(n_sheets);
    for (int s = 0; s < n_sheets; s++) {
        const cs_material_desc& m = mats[sheets[s].material];
        std::vector<float> rows(&m.stretching[0][0], &m.stretching[0][0] + 24);
        float smult = m.stretching_mult * m.thicken;
        std::vector<float> key = rows;
        key.push_back(smult);
        auto it = tableIndex.find(key);
        if (it != tableIndex.end()) {
            sheetTable[s] = it->second;
            continue;
        }
        auto bt = baseSamples.find(rows);
        if (bt == baseSamples.end()) bt = baseSamples.emplace(rows, stretchingSamples(m.stretching)).first;
        int id = (int)(tables.size() / CS_TABLE_ENTRIES);
        tableIndex[key] = id;
        sheetTable[s] = id;
        const std::vector<float>& b = bt->second;
        for (int i = 0; i < CS_TABLE_ENTRIES; i++)
            tables.push_back(make_float4(b[4 * i] * smult, b[4 * i + 1] * smult, b[4 * i + 2] * smult, b[4 * i + 3] * smult));
    }

    // per-sheet arrays
    Batch& B = c->B;
    std::vector<float> hx, hv, hmass;
    std::vector<float4> hhandle, hface_inv, hedge_par;
    std::vector<int4> hface_nodes, hedge_nodes;
    std::vector<float> hface_area;
    std::vector<int> hedge_meta, hedge_sheet;
    std::vector<SheetDesc> hs(n_sheets);
    std::vector<SliceDesc> hslices;
    // per-topology arrays, concatenated
    std::vector<int> htcol, hrface_ptr, hredge_ptr;
    std::vector<int2> hrface, hredge;
    int gatherWidth = 1;
    std::vector<int> hnbr_ptr, hnbr, hnode_sheet, hrowmap, hrow2slot;
    std::vector<int> topoRow2Slot0(topos.size());
    std::vector<int> topoNbrPtr0(topos.size()), topoNbr0(topos.size());
    std::vector<int> topoPanel0(topos.size()), topoSlice0(topos.size());
    std::vector<int> htcsr_ptr, htcsr_col, htcsr_slot, topoCsrPtr0(topos.size());
    // Cluster-resident solve plan (resident.cu).  Clusters must fit a GPC, so the number of
    // SMs a cluster size keeps busy varies: 8- and 9-CTA clusters are planned and the one that
    // makes the most sheets resident, then keeps the most SMs busy, is taken (on the B200, 15
    // clusters of 8 occupy 120 SMs, 15 clusters of 9 occupy 135, 11 of 10 occupy 110).
    // CS_RESIDENT_CL (2..16) forces a size; 0 solves every sheet in the batched loop.
    std::vector<int> candidates = {8, 9, 10};
    if (const char* ev = std::getenv("CS_RESIDENT_CL")) {
        const int v = std::atoi(ev);
        if (v != 0 && (v < 2 || v > CS_RES_MAX_CL))
            return fail(c, CS_ERR_INVALID_ARG, "CS_RESIDENT_CL must be 0 or 2..16");
        candidates = {v};
    }
    struct ResChoice {
        int cl = 0, w = 0, panels = 0, halo = 0, cap = 0, clusters = 0, ck = 0;
        long long sheets = 0;
        size_t smem = 0;
        std::vector<ResidentPlan> plans;
        std::vector<char> resident;
    };
    cudaDeviceProp devProp;
    CS_CUDA(cudaGetDeviceProperties(&devProp, c->device));
    cudaFuncAttributes resAttr;
    CS_CUDA(cudaFuncGetAttributes(&resAttr, cs_resident_pcg_kernel));
    auto planFor = [&](int cl) {
        ResChoice R;
        R.cl = cl;
        R.plans.resize(topos.size());
        R.resident.assign(topos.size(), 0);
        for (size_t t = 0; t < topos.size() && cl > 0; t++) {
            R.plans[t] = residentPlan(*topos[t], cl);
            const ResidentPlan& P = R.plans[t];
            // p indices (own slots + halo) are 12-bit in the kernel's packed column codes
            if (P.w > CS_RES_MAX_WARPS || P.max_width > CS_RES_MAX_WIDTH || P.max_halo + CS_RES_MAX_WARPS * CS_SLICE >= 4096)
                continue;
            R.resident[t] = 1;
            R.w = std::max(R.w, P.w);
            R.panels = std::max(R.panels, P.max_panels);
            R.halo = std::max(R.halo, P.max_halo);
        }
        if (R.w == 0) return R;
        // coarse-space correction for the topologies with the strip-local Chebyshev
        // preconditioner (it needs a second warp for the segment sums)
        R.ck = coarseSegments(cl);
        bool anyCoarse = false;
        for (size_t t = 0; t < topos.size(); t++)
            anyCoarse |= R.resident[t] && R.plans[t].blocks > 0 &&
                         (double)R.plans[t].local_blocks >= CS_CHEB_MIN_LOCAL * (double)R.plans[t].blocks;
        if (!anyCoarse || R.ck < 2 || R.w < 2) R.ck = 0;
        // p array: own slots, halo slots, then a second own-slot buffer (strip-local Chebyshev),
        // then the coarse region
        const size_t ubytes = ((size_t)2 * R.w * CS_SLICE + R.halo) * sizeof(float4);
        const size_t pbytes = ubytes + coarseSmemBytes(cl, R.ck);
        const size_t budget = devProp.sharedMemPerBlockOptin > resAttr.sharedSizeBytes + pbytes
                                  ? devProp.sharedMemPerBlockOptin - resAttr.sharedSizeBytes - pbytes : 0;
        R.cap = (int)std::min<size_t>((size_t)R.panels, budget / (CS_PANEL_FLOATS * sizeof(float)));
        R.smem = (size_t)R.cap * CS_PANEL_FLOATS * sizeof(float) + pbytes;
        if (budget > 0) {
            raiseDynSmem((const void*)cs_resident_pcg_kernel, R.smem);
            if (cl > 8) cudaFuncSetAttribute(cs_resident_pcg_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = cl;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(cl);
            cfg.blockDim = dim3(R.w * CS_SLICE);
            cfg.dynamicSmemBytes = R.smem;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            if (cudaOccupancyMaxActiveClusters(&R.clusters, cs_resident_pcg_kernel, &cfg) != cudaSuccess) R.clusters = 0;
            cudaGetLastError();
        }
        if (R.clusters <= 0) {
            R.clusters = 0;
            std::fill(R.resident.begin(), R.resident.end(), 0);
        }
        for (int sh = 0; sh < n_sheets; sh++) R.sheets += R.resident[sheetTopoId[sh]];
        return R;
    };
    ResChoice res;
    for (int cl : candidates) {
        ResChoice R = planFor(cl);
        const bool better = res.cl == 0 || R.sheets > res.sheets ||
                            (R.sheets == res.sheets && (long long)R.clusters * R.cl > (long long)res.clusters * res.cl);
        if (better) res = std::move(R);
    }
    std::vector<int> hrsplit(topos.size() * (CS_RES_MAX_CL + 1), 0), hrcode;
    std::vector<int> hrsendptr(topos.size() * (CS_RES_MAX_CL + 1), 0);
    std::vector<int> hrhalo(topos.size() * (CS_RES_MAX_CL + 1), 0);
    // sheets whose strips keep enough of the couplings use the strip-local Chebyshev
    // preconditioner (when asked for); the others stay with block-Jacobi
    std::vector<int> hrcheb(topos.size() * (CS_RES_MAX_CL + 1), 0);
    std::vector<uint32_t> hrsend;
    std::vector<char>& topoResident = res.resident;
    std::vector<ResidentPlan>& plans = res.plans;
    const int resW = res.w, resCap = res.cap;
    for (size_t t = 0; t < topos.size(); t++)
        if (topoResident[t]) {
            std::copy(plans[t].split.begin(), plans[t].split.end(), hrsplit.begin() + t * (CS_RES_MAX_CL + 1));
            std::copy(plans[t].halo_count.begin(), plans[t].halo_count.end(), hrhalo.begin() + t * (CS_RES_MAX_CL + 1));
            const bool cheb = plans[t].blocks > 0 &&
                              (double)plans[t].local_blocks >= CS_CHEB_MIN_LOCAL * (double)plans[t].blocks;
            for (int r = 0; r <= CS_RES_MAX_CL; r++) hrcheb[t * (CS_RES_MAX_CL + 1) + r] = cheb;
            if (cheb && res.ck > 0) {
                // segments, then the lanes of each slice grouped by segment, then the plans
                // again over the moved slots (the slices and their rows stay)
                coarsePlan(*topos[t], plans[t], res.cl, res.ck);
                permuteLanesByAggregate(*topos[t], plans[t].coarse.agg);
                plans[t] = residentPlan(*topos[t], res.cl);
                coarsePlan(*topos[t], plans[t], res.cl, res.ck);
            }
        }
    // coarse-space arrays, per topology concatenated
    std::vector<int4> hrcoarse(topos.size(), make_int4(0, 0, 0, 0)), hcpair;
    std::vector<int> hragg, hrwmask(topos.size() * CS_RES_MAX_CL * CS_RES_MAX_WARPS, 0), hccontrib;
    for (size_t t = 0; t < topos.size(); t++) {
        static const CoarsePlan none;
        const CoarsePlan& C = t < plans.size() ? plans[t].coarse : none;
        if (topoResident[t] && C.nc > 0) {
            const int p0 = (int)hcpair.size(), c0 = (int)hccontrib.size();
            for (const int4& q : C.pairs) hcpair.push_back(make_int4(q.x, q.y, q.z + c0, q.w + c0));
            hccontrib.insert(hccontrib.end(), C.contrib.begin(), C.contrib.end());
            std::copy(C.wmask.begin(), C.wmask.end(), hrwmask.begin() + t * CS_RES_MAX_CL * CS_RES_MAX_WARPS);
            hrcoarse[t] = make_int4(C.nc, C.K, p0, (int)hcpair.size());
            hragg.insert(hragg.end(), C.agg.begin(), C.agg.end());
        } else {
            hragg.insert(hragg.end(), topos[t]->n_nodes, -1);
        }
    }
    // the batched loop's coarse spaces (after the lane moves above: the contributor slots refer
    // to the final slot numbering); up to CS_BC_MAX_G^2 aggregates when 16-CTA clusters can run
    // the larger inversions, else as many as one CTA inverts
    int bcGmax = CS_BC_MAX_G;
    {
        const size_t nblkMax = (CS_BC_MAX_NC + CS_BC_KB - 1) / CS_BC_KB;
        const size_t rm = CS_BC_KB * ((nblkMax + CS_BC_CLUSTER - 1) / CS_BC_CLUSTER);
        const size_t ub = ((size_t)CS_BC_KB * CS_BC_MAX_NC + 1 + 3) & ~(size_t)3;
        const size_t smemBig =
            (((rm * CS_BC_MAX_NC + 3) & ~(size_t)3) + ub + rm * CS_BC_KB + CS_BC_KB * CS_BC_KB) * sizeof(float);
        int nclusters = 0;
        if (cudaFuncSetAttribute(cs_bc_invert_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBig) ==
                cudaSuccess &&
            cudaFuncSetAttribute(cs_bc_invert_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
                cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = CS_BC_CLUSTER;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(CS_BC_CLUSTER);
            cfg.blockDim = dim3(CS_BC_THREADS);
            cfg.dynamicSmemBytes = smemBig;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            if (cudaOccupancyMaxActiveClusters(&nclusters, cs_bc_invert_cluster_kernel, &cfg) != cudaSuccess) nclusters = 0;
        }
        cudaGetLastError();
        c->bcSmemBig = smemBig;
        if (nclusters <= 0) bcGmax = 8;  // 64 aggregates, 192 unknowns: one CTA inverts them
        CS_CUDA(cudaFuncSetAttribute(cs_bc_invert_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (CS_BC_SMALL_NC * CS_BC_SMALL_NC + 4 + 2 * CS_BC_KB * CS_BC_SMALL_NC + CS_BC_KB * CS_BC_KB) * (int)sizeof(float)));
    }
    std::vector<BCPlan> bcplans(topos.size());
    for (size_t t = 0; t < topos.size(); t++) batchedCoarsePlan(*topos[t], bcGmax, bcplans[t]);
    std::vector<int> hbc_node_agg, hbc_mptr, hbc_mem, hbc_contrib;
    std::vector<int4> hbc_pair;
    std::vector<int> topoBcNode0(topos.size()), topoBcAgg0(topos.size()), topoBcMem0(topos.size()),
        topoBcPair0(topos.size());
    for (size_t t = 0; t < topos.size(); t++) {
        const BCPlan& P = bcplans[t];
        topoBcNode0[t] = (int)hbc_node_agg.size();
        topoBcAgg0[t] = (int)hbc_mptr.size();
        topoBcMem0[t] = (int)hbc_mem.size();
        topoBcPair0[t] = (int)hbc_pair.size();
        hbc_node_agg.insert(hbc_node_agg.end(), P.agg.begin(), P.agg.end());
        hbc_mptr.insert(hbc_mptr.end(), P.mptr.begin(), P.mptr.end());
        hbc_mem.insert(hbc_mem.end(), P.mem.begin(), P.mem.end());
        const int c0 = (int)hbc_contrib.size();
        for (const int4& q : P.pairs) hbc_pair.push_back(make_int4(q.x, q.y, q.z + c0, q.w + c0));
        hbc_contrib.insert(hbc_contrib.end(), P.contrib.begin(), P.contrib.end());
    }
    c->resCL = c->resThreads = c->resClusters = 0;
    c->resSmem = 0;
    B.res_cnc = B.res_ck = B.res_coff = 0;
    if (res.clusters > 0 && res.ck > 0) {
        B.res_ck = res.ck;
        B.res_cnc = 3 * res.cl * res.ck;
        B.res_coff = (int)(res.smem - coarseSmemBytes(res.cl, res.ck));
        CS_CUDA(raiseDynSmem((const void*)cs_coarse_setup_kernel, cs_coarse_setup_smem(B.res_cnc)));
    }
    if (res.clusters > 0) {
        // the launch attributes of the chosen plan (the evaluation set others)
        CS_CUDA(raiseDynSmem((const void*)cs_resident_pcg_kernel, res.smem));
        c->resCL = res.cl;
        c->resThreads = resW * CS_SLICE;
        c->resClusters = res.clusters;
        c->resSmem = res.smem;
    }
    {
        int tp = 0, ts = 0;
        for (size_t t = 0; t < topos.size(); t++) {
            topoPanel0[t] = tp;
            topoSlice0[t] = ts;
            const Topo& T = *topos[t];
            htcol.insert(htcol.end(), T.tcol.begin(), T.tcol.end());
            if (topoResident[t]) {
                // halo slots follow the batch's own slots in every CTA's p array
                for (int code : plans[t].code)
                    hrcode.push_back(code & CS_RES_HALO_BIT ? resW * CS_SLICE + (code & ~CS_RES_HALO_BIT) : code);
                const int base = (int)hrsend.size();
                for (int k = 0; k <= CS_RES_MAX_CL; k++) hrsendptr[t * (CS_RES_MAX_CL + 1) + k] = base + plans[t].sendptr[k];
                hrsend.insert(hrsend.end(), plans[t].send.begin(), plans[t].send.end());
            } else {
                hrcode.insert(hrcode.end(), T.tcol.size(), 0);
            }
            // the gather's row lists at the row2slot offsets (node-indexed; the next topology's
            // first pointer ends this one's last row)
            for (int i = 0; i < T.n_nodes; i++) hrface_ptr.push_back(T.rf_ptr[i] + (int)hrface.size());
            for (int i = 0; i < T.n_nodes; i++) hredge_ptr.push_back(T.re_ptr[i] + (int)hredge.size());
            hrface.insert(hrface.end(), T.rf.begin(), T.rf.end());
            hredge.insert(hredge.end(), T.re.begin(), T.re.end());
            for (int w : T.slice_width) gatherWidth = std::max(gatherWidth, w);
            hrowmap.insert(hrowmap.end(), T.rowmap.begin(), T.rowmap.end());
            topoRow2Slot0[t] = (int)hrow2slot.size();
            hrow2slot.insert(hrow2slot.end(), T.row2slot.begin(), T.row2slot.end());
            topoCsrPtr0[t] = (int)htcsr_ptr.size();
            for (int v : T.csr_ptr) htcsr_ptr.push_back(v + (int)htcsr_col.size());
            htcsr_col.insert(htcsr_col.end(), T.csr_col.begin(), T.csr_col.end());
            htcsr_slot.insert(htcsr_slot.end(), T.csr_slot.begin(), T.csr_slot.end());
            topoNbrPtr0[t] = (int)hnbr_ptr.size();
            topoNbr0[t] = (int)hnbr.size();
            hnbr_ptr.insert(hnbr_ptr.end(), T.nbr_ptr.begin(), T.nbr_ptr.end());
            hnbr.insert(hnbr.end(), T.nbr.begin(), T.nbr.end());
            tp += T.n_tpanels;
            ts += T.n_slices;
        }
        hrface_ptr.push_back((int)hrface.size());
        hredge_ptr.push_back((int)hredge.size());
        if (hrface.empty()) hrface.push_back(make_int2(0, 0));
        if (hredge.empty()) hredge.push_back(make_int2(0, 0));
    }
    int node_off = 0, face_off = 0, edge_off = 0, slice_off = 0, panel_off = 0;
    long long nnzb = 0;
    int bcVec = 0, bcMaxPair = 0;
    long long bcMat = 0;
    std::vector<int2> hbc_agg;
    std::vector<int> hbc_big;
    for (int s = 0; s < n_sheets; s++) {
        const cs_sheet_desc& d = sheets[s];
        const cs_material_desc& m = mats[d.material];
        const Topo& T = *topos[sheetTopoId[s]];
        SheetDesc& sd = hs[s];
        sd.node_off = node_off;
        sd.n_nodes = d.n_nodes;
        sd.face_off = face_off;
        sd.n_faces = d.n_faces;
        sd.edge_off = edge_off;
        sd.n_edges = (int)T.ie_meta.size();
        sd.slice_off = slice_off;
        sd.n_slices = T.n_slices;
        sd.topo = sheetTopoId[s];
        sd.table = sheetTable[s];
        sd.nbr_ptr_off = topoNbrPtr0[sheetTopoId[s]];
        sd.row2slot_off = topoRow2Slot0[sheetTopoId[s]];
        sd.nbr_off = topoNbr0[sheetTopoId[s]];
        sd.resident = topoResident[sheetTopoId[s]];
        sd.csr_ptr_off = topoCsrPtr0[sheetTopoId[s]];
        sd.panel_off = panel_off;
        {
            const int t = sheetTopoId[s];
            const BCPlan& P = bcplans[t];
            sd.bc_node_off = topoBcNode0[t];
            sd.bc_agg_off = topoBcAgg0[t];
            sd.bc_mem_off = topoBcMem0[t];
            sd.bc_pair_off = topoBcPair0[t];
            sd.bc_npair = (int)P.pairs.size();
            sd.bc_na = P.na;
            sd.bc_vec_off = bcVec;
            sd.bc_mat_off = bcMat;
            bcVec += 3 * P.na;
            bcMat += (long long)(3 * P.na) * (3 * P.na);
            for (int a = 0; a < P.na; a++) hbc_agg.push_back(make_int2(s, a));
            if (3 * P.na > CS_BC_SMALL_NC) hbc_big.push_back(s);
            bcMaxPair = std::max(bcMaxPair, (int)P.pairs.size());
        }
        hnode_sheet.insert(hnode_sheet.end(), d.n_nodes, s);
        float bmult = m.bending_mult * m.thicken;
        for (int i = 0; i < 15; i++) sd.bending[i] = m.bending[i / 5][i % 5] * bmult;
        sd.wind_density = d.wind_density;
        sd.wind_drag = d.wind_drag;
        for (int i = 0; i < 3; i++) sd.wind_v[i] = d.wind_velocity[i];
        float density = m.density * (m.density_mult * m.thicken);
        // nodes
        for (int i = 0; i < 3 * d.n_nodes; i++) {
            hx.push_back(d.x[i]);
            hv.push_back(d.v ? d.v[i] : 0.0f);
        }
        // faces: Face::initialize (Face.cu:12-20)
        std::vector<float> fmass(d.n_faces);
        for (int f = 0; f < d.n_faces; f++) {
            const float* u0 = d.uv + 2 * d.face_verts[3 * f];
            const float* u1 = d.uv + 2 * d.face_verts[3 * f + 1];
            const float* u2 = d.uv + 2 * d.face_verts[3 * f + 2];
            float d1x = u1[0] - u0[0], d1y = u1[1] - u0[1], d2x = u2[0] - u0[0], d2y = u2[1] - u0[1];
            float a = d1x, b = d2x, cc = d1y, dd = d2y;
            float invDet = 1.0f / (a * dd - b * cc);
            float4 inv = make_float4(dd * invDet, -b * invDet, -cc * invDet, a * invDet);
            float cr = d1x * d2y - d1y * d2x;
            float area = 0.5f * (cr < 0.0f ? -cr : cr);
            if (!(area > 0.0f)) return fail(c, CS_ERR_INVALID_ARG, "sheet %d face %d: zero rest area", s, f);
            hface_inv.push_back(inv);
            hface_area.push_back(area);
            fmass[f] = area * density;
            hface_nodes.push_back(make_int4(node_off + d.face_nodes[3 * f], node_off + d.face_nodes[3 * f + 1],
                                            node_off + d.face_nodes[3 * f + 2], s));
        }
        // lumped mass (Mesh.cu:190-200)
        std::vector<float> mass(d.n_nodes, 0.0f);
        for (int f = 0; f < d.n_faces; f++) {
            float mm = fmass[f] / 3.0f;
            for (int k = 0; k < 3; k++) mass[d.face_nodes[3 * f + k]] += mm;
        }
        hmass.insert(hmass.end(), mass.begin(), mass.end());
        // handles
        std::vector<float4> hd(d.n_nodes, make_float4(0.f, 0.f, 0.f, 0.f));
        for (int h = 0; h < d.n_handles; h++) {
            int i = d.handle_nodes[h];
            const float* p = d.handle_pos ? d.handle_pos + 3 * h : d.x + 3 * i;
            c->handleNode.push_back(node_off + i);
            hd[i] = make_float4(p[0], p[1], p[2], hd[i].w + 1.0f);
        }
        hhandle.insert(hhandle.end(), hd.begin(), hd.end());
        // interior edges
        for (size_t e = 0; e < T.ie_meta.size(); e++) {
            const int* n4 = &T.ie_nodes[4 * e];
            hedge_nodes.push_back(make_int4(node_off + n4[0], node_off + n4[1], node_off + n4[2], node_off + n4[3]));
            hedge_meta.push_back(T.ie_meta[e]);
            hedge_sheet.push_back(s);
            int f0 = T.ie_faces[2 * e], f1 = T.ie_faces[2 * e + 1];
            float area = hface_area[face_off + f0] + hface_area[face_off + f1];
            const int* ev = &T.ie_verts[4 * e];
            float b0 = biasWeight(d.uv[2 * ev[1]] - d.uv[2 * ev[0]], d.uv[2 * ev[1] + 1] - d.uv[2 * ev[0] + 1]);
            float b1 = biasWeight(d.uv[2 * ev[3]] - d.uv[2 * ev[2]], d.uv[2 * ev[3] + 1] - d.uv[2 * ev[2] + 1]);
            hedge_par.push_back(make_float4(area, b0, b1, 0.0f));
        }
        // slices
        for (int t = 0; t < T.n_slices; t++) {
            SliceDesc sl{};
            sl.sheet = s;
            sl.topo_slice = topoSlice0[sheetTopoId[s]] + t;
            sl.row0 = node_off;  // rows: row0 + rowmap[topo_slice * 32 + lane]
            sl.rows = T.slice_rows[t];
            sl.width = T.slice_width[t];
            sl.panel0 = panel_off + T.slice_tpanel0[t];
            sl.tpanel0 = topoPanel0[sheetTopoId[s]] + T.slice_tpanel0[t];
            hslices.push_back(sl);
        }
        node_off += d.n_nodes;
        face_off += d.n_faces;
        edge_off += (int)T.ie_meta.size();
        slice_off += T.n_slices;
        panel_off += T.n_tpanels;
        nnzb += T.nnzb;
    }
    B.N = node_off;
    B.F = face_off;
    B.E = edge_off;
    B.S = n_sheets;
    B.n_slices = slice_off;
    B.n_panels = panel_off;
    B.n_tpanels = (int)(htcol.size() / CS_SLICE);
    B.n_tables = (int)(tables.size() / CS_TABLE_ENTRIES);
    c->nnzb_pattern = nnzb;
    // resident sheets, largest first (the persistent clusters take them in this order)
    std::vector<int> hrlist;
    for (int s = 0; s < n_sheets; s++)
        if (hs[s].resident) hrlist.push_back(s);
    std::stable_sort(hrlist.begin(), hrlist.end(), [&](int a, int b) { return hs[a].n_slices > hs[b].n_slices; });
    B.n_resident = (int)hrlist.size();
    B.res_cap = resCap;
    B.res_halo0 = resW * CS_SLICE;
    B.res_alt = resW * CS_SLICE + res.halo;
    c->resClustersMax = c->resClusters;
    c->resClusters = std::min(c->resClusters, B.n_resident);
    c->rlistAll = hrlist;
    c->rlistCur = hrlist;
    c->sheetBlocks.assign(n_sheets, 0);
    c->sheetLocalBlocks.assign(n_sheets, 0);
    for (int s : hrlist) {
        c->sheetBlocks[s] = plans[sheetTopoId[s]].blocks;
        c->sheetLocalBlocks[s] = plans[sheetTopoId[s]].local_blocks;
    }
    c->sheets = hs;
    c->slices = hslices;

    cs_status st;
#define UP(field, vec) \
    if ((st = upload(c, &B.field, vec)) != CS_OK) return st;
    UP(x, hx);
    UP(v, hv);
    UP(mass, hmass);
    UP(handle, hhandle);
    UP(handle_motion, std::vector<int>(hhandle.size(), -1));
    c->maxHandleMotion = -1;
    UP(face_nodes, hface_nodes);
    UP(face_inv, hface_inv);
    UP(face_area, hface_area);
    UP(edge_nodes, hedge_nodes);
    UP(edge_meta, hedge_meta);
    UP(edge_sheet, hedge_sheet);
    UP(edge_par, hedge_par);
    UP(sheets, hs);
    UP(tables, tables);
    UP(slices, hslices);
    UP(tcol, htcol);
    UP(rface_ptr, hrface_ptr);
    UP(redge_ptr, hredge_ptr);
    UP(rface, hrface);
    UP(redge, hredge);
    B.gather_width = gatherWidth;
    UP(nbr_ptr, hnbr_ptr);
    UP(nbr, hnbr);
    UP(node_sheet, hnode_sheet);
    UP(rowmap, hrowmap);
    UP(bc_agg, hbc_agg);
    UP(bc_big, hbc_big);
    UP(bc_node_agg, hbc_node_agg);
    UP(bc_mptr, hbc_mptr);
    UP(bc_mem, hbc_mem);
    UP(bc_pair, hbc_pair);
    UP(bc_contrib, hbc_contrib);
    if ((st = dalloc(c, &B.bc_mat, (size_t)std::max(1LL, bcMat))) != CS_OK) return st;
    if ((st = dalloc(c, &B.bc_inv, (size_t)std::max(1LL, bcMat))) != CS_OK) return st;
    if ((st = dalloc(c, &B.bc_rc, (size_t)std::max(1, bcVec))) != CS_OK) return st;
    if ((st = dalloc(c, &B.bc_ec, (size_t)std::max(1, bcVec))) != CS_OK) return st;
    UP(bc_ok, std::vector<int>(n_sheets, 0));
    B.bc_total_agg = (int)hbc_agg.size();
    B.bc_max_npair = bcMaxPair;
    B.bc_n_big = (int)hbc_big.size();
    c->bcMatFloats = bcMat;
    UP(row2slot, hrow2slot);
    UP(tcsr_ptr, htcsr_ptr);
    UP(tcsr_col, htcsr_col);
    UP(tcsr_slot, htcsr_slot);
    UP(rlist, hrlist);
    UP(rsplit, hrsplit);
    UP(rcode, hrcode);
    UP(rsendptr, hrsendptr);
    UP(rsend, hrsend);
    UP(rhalo, hrhalo);
    UP(rcheb, hrcheb);
    UP(rcoarse, hrcoarse);
    UP(ragg, hragg);
    UP(rwmask, hrwmask);
    UP(cpair, hcpair);
    UP(ccontrib, hccontrib);
#undef UP
#define AL(field, n) \
    if ((st = dalloc(c, &B.field, (size_t)(n))) != CS_OK) return st;
    AL(dv, 3LL * B.N);
    AL(x0, 3LL * B.N);
    AL(edge_geo, 4LL * std::max(B.E, 1));
    AL(dv64, 3LL * B.N);
    AL(warm, 3LL * B.N);
    AL(A, (long long)B.n_panels * CS_PANEL_FLOATS);
    AL(b, 3LL * B.N);
    AL(Pinv, 9LL * B.N);
    AL(e, 3LL * B.N);
    AL(r, 3LL * B.N);
    AL(z, 3LL * B.N);
    AL(pA, 3LL * B.N);
    AL(pB, 3LL * B.N);
    AL(q, 3LL * B.N);
    AL(part, 2LL * B.n_slices);
    AL(inst, B.S);
    AL(params, 1);
    AL(loop, 8);
    AL(cinv, B.res_cnc > 0 ? (long long)hrlist.size() * B.res_cnc * B.res_cnc : 1);
    AL(cvalid, std::max<size_t>(hrlist.size(), 1));
#undef AL
    CS_CUDA(cudaMemset(B.dv, 0, 3LL * B.N * sizeof(float)));
    CS_CUDA(cudaMemcpy(B.x0, B.x, 3LL * B.N * sizeof(float), cudaMemcpyDeviceToDevice));  // Node::Node
    CS_CUDA(cudaMemset(B.warm, 0, 3LL * B.N * sizeof(float)));
    CS_CUDA(cudaMemset(B.A, 0, (size_t)B.n_panels * CS_PANEL_FLOATS * sizeof(float)));
    CS_CUDA(cudaMemset(B.inst, 0, B.S * sizeof(InstState)));
    CS_CUDA(cudaMemset(B.loop, 0, 8 * sizeof(int)));
    CS_CUDA(cudaDeviceSynchronize());
    {
        cudaDeviceProp prop;
        CS_CUDA(cudaGetDeviceProperties(&prop, c->device));
        // persistent gather: CTAs of up to CS_GATHER_THREADS / 32 warps, fewer when a warp's
        // slot accumulators (the widest slice's slots x 1,152 bytes) would not fit four times in
        // a CTA's shared memory (meshes with high-valence nodes); as many CTAs per SM as the
        // accumulators allow (at most CS_GATHER_CTAS_PER_SM, 1..16, when set)
        const size_t perWarp = (size_t)B.gather_width * 9 * CS_SLICE * sizeof(float);
        c->gatherWarps = (int)std::min<size_t>(CS_GATHER_THREADS / 32, (size_t)prop.sharedMemPerBlockOptin / perWarp);
        if (c->gatherWarps < 1)
            return fail(c, CS_ERR_INVALID_ARG, "slices of %d block slots exceed the assembly's shared memory", B.gather_width);
        c->gatherSmem = (size_t)c->gatherWarps * perWarp;
        CS_CUDA(raiseDynSmem((const void*)cs_gather_kernel, c->gatherSmem));
        const int threads = 32 * c->gatherWarps;
        int perSM = 0;
        CS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, cs_gather_kernel, threads, c->gatherSmem));
        if (const char* ev = std::getenv("CS_GATHER_CTAS_PER_SM")) perSM = std::min(perSM, std::min(16, std::max(1, std::atoi(ev))));
        perSM = std::max(perSM, 1);
        c->gatherGrid = std::max(1, std::min(nblk((long long)B.n_slices * 32, threads), perSM * prop.multiProcessorCount));
    }
    c->loaded = true;
    return CS_OK;
}

cs_status cs_get_solver_info(const cs_ctx* c, int* info) {
    if (!c || !info) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return CS_ERR_STATE;
    info[0] = c->B.n_resident;
    info[1] = c->resCL;
    info[2] = c->resThreads;
    info[3] = c->resClusters;
    info[4] = c->B.res_cap;
    info[5] = (int)c->resSmem;
    info[6] = kSpmvShapes[c->spmvShape].threads;
    info[7] = kSpmvShapes[c->spmvShape].spw;
    info[8] = kSpmvShapes[c->spmvShape].unroll;
    info[9] = c->tunedDegree;
    info[10] = c->tunedCoarse;
    return CS_OK;
}

cs_status cs_get_resident_blocks(const cs_ctx* c, long long* out) {
    if (!c || !out) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return CS_ERR_STATE;
    out[0] = out[1] = 0;
    for (int s : c->rlistCur) {
        out[0] += c->sheetBlocks[s];
        out[1] += c->sheetLocalBlocks[s];
    }
    out[2] = CS_CHEB_POWER_ITERS;
    return CS_OK;
}

cs_status cs_get_sizes(const cs_ctx* c, long long* sizes) {
    if (!c || !sizes) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return CS_ERR_STATE;
    sizes[0] = c->B.N;
    sizes[1] = c->B.F;
    sizes[2] = c->B.E;
    sizes[3] = (long long)c->B.n_panels * CS_SLICE;
    sizes[4] = c->B.n_slices;
    sizes[5] = c->B.S;
    sizes[6] = c->nnzb_pattern + c->B.n_px;
    return CS_OK;
}

cs_status cs_set_state(cs_ctx* c, const float* x, const float* v) {
    if (!c || (!x && !v)) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    size_t n = 3 * (size_t)c->B.N * sizeof(float);
    if (x) CS_CUDA(cudaMemcpyAsync(c->B.x, x, n, cudaMemcpyHostToDevice, c->stream));
    if (v) CS_CUDA(cudaMemcpyAsync(c->B.v, v, n, cudaMemcpyHostToDevice, c->stream));
    return CS_OK;
}

}  // extern "C"

namespace {

void destroyGraphs(cs_ctx* c) {
    for (int l = 0; l < 2; l++)
        for (int k = 0; k < 2; k++) {
            if (c->gexec[l][k]) cudaGraphExecDestroy(c->gexec[l][k]);
            if (c->gph[l][k]) cudaGraphDestroy(c->gph[l][k]);
            c->gexec[l][k] = nullptr;
            c->gph[l][k] = nullptr;
        }
}

template <class T>
cs_status grow(cs_ctx* c, T*& p, size_t& cap, size_t need) {
    if (need <= cap && p) return CS_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t n = std::max<size_t>(need + need / 4, 16);
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) return fail(c, CS_ERR_CUDA, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    cap = n;
    return CS_OK;
}

// Exclusive scan of n ints on the device, in place; data[n] receives the total (and *total,
// when given, after a stream synchronisation).
cs_status scanInts(cs_ctx* c, int* data, int n, int* total) {
    ProxBuffers& P = c->prox;
    const int nb = std::max(1, (n + CS_SCAN_ITEMS - 1) / CS_SCAN_ITEMS);
    cs_status st;
    if ((st = grow(c, P.partial, P.partialCap, nb)) != CS_OK) return st;
    cs_scan_sums_kernel<<<nb, 1024, 0, c->stream>>>(data, n, P.partial);
    cs_scan_partials_kernel<<<1, 1024, 0, c->stream>>>(P.partial, nb, data + n);
    cs_scan_apply_kernel<<<nb, 1024, 0, c->stream>>>(data, n, P.partial);
    CS_CUDA(cudaGetLastError());
    if (total) {
        CS_CUDA(cudaMemcpyAsync(total, data + n, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CS_CUDA(cudaStreamSynchronize(c->stream));
    }
    return CS_OK;
}

void clearProximities(cs_ctx* c) {
    Batch& B = c->B;
    B.n_pinst = B.n_px = 0;
    B.pinst = nullptr;
    B.prec = nullptr;
    B.prow_ptr = B.prow_inst = nullptr;
    B.xptr = B.xcol = nullptr;
    B.xval = nullptr;
    B.sheet_prox = nullptr;
    c->prox.n = 0;
}

// The proximities in prox.desc (n on the device) become the terms of the following steps:
// one instance per (proximity, sheet holding one of its nodes) in proximity order, per-row
// instance lists and the outside-pattern side list, all built on the device (proxlist.cu);
// cs_prox_row_kernel then adds the terms in the reference's order (Cloth.cu:171-192).
cs_status applyProximities(cs_ctx* c, int n, float thickness) {
    Batch& B = c->B;
    ProxBuffers& P = c->prox;
    if (n == 0 && P.n == 0 && B.n_pinst == 0) return CS_OK;  // none before, none now: nothing changes
    destroyGraphs(c);  // the captured launches hold the old lists
    clearProximities(c);
    std::vector<int> touched(B.S, 0);
    cs_status st;
    if (n > 0) {
        const size_t N1 = (size_t)B.N + 1;
        if ((st = grow(c, P.icount, P.icountCap, (size_t)n + 1)) != CS_OK) return st;
        cs_prox_count_kernel<<<nblk(n, 128), 128, 0, c->stream>>>(B, P.desc, n, P.icount);
        int T = 0;
        if ((st = scanInts(c, P.icount, n, &T)) != CS_OK) return st;
        if ((st = grow(c, P.inst, P.instCap, (size_t)T)) != CS_OK) return st;
        if ((st = grow(c, P.rec, P.recCap, (size_t)T * CS_PROX_REC)) != CS_OK) return st;
        if ((st = grow(c, P.sheetProx, P.sheetCap, (size_t)B.S)) != CS_OK) return st;
        CS_CUDA(cudaMemsetAsync(P.sheetProx, 0, B.S * sizeof(int), c->stream));
        cs_prox_expand_kernel<<<nblk(n, 128), 128, 0, c->stream>>>(B, P.desc, n, P.icount, thickness, P.inst,
                                                                     P.sheetProx);
        if ((st = grow(c, P.rowPtr, P.rowCap, N1)) != CS_OK) return st;
        if ((st = grow(c, P.rowFill, P.rowFillCap, N1)) != CS_OK) return st;
        if ((st = grow(c, P.xptr, P.xptrCap, N1)) != CS_OK) return st;
        CS_CUDA(cudaMemsetAsync(P.rowPtr, 0, N1 * sizeof(int), c->stream));
        CS_CUDA(cudaMemsetAsync(P.rowFill, 0, N1 * sizeof(int), c->stream));
        cs_prox_rowcount_kernel<<<nblk(T, 128), 128, 0, c->stream>>>(P.inst, T, P.rowPtr);
        int L = 0;
        if ((st = scanInts(c, P.rowPtr, B.N, &L)) != CS_OK) return st;
        if ((st = grow(c, P.rowInst, P.rowInstCap, (size_t)L)) != CS_OK) return st;
        cs_prox_rowfill_kernel<<<nblk(T, 128), 128, 0, c->stream>>>(P.inst, T, P.rowPtr, P.rowFill, P.rowInst);
        cs_prox_rowsort_kernel<<<nblk(B.N, 128), 128, 0, c->stream>>>(B.N, P.rowPtr, P.rowInst);
        // the lists cs_prox_outside_kernel reads through B
        B.prow_ptr = P.rowPtr;
        B.prow_inst = P.rowInst;
        cs_prox_outside_kernel<<<nblk(B.N, 128), 128, 0, c->stream>>>(B, P.rowPtr, P.rowInst, P.inst, nullptr, P.xptr);
        int X = 0;
        if ((st = scanInts(c, P.xptr, B.N, &X)) != CS_OK) return st;
        if (X > 0) {
            if ((st = grow(c, P.xcol, P.xcolCap, (size_t)X)) != CS_OK) return st;
            if ((st = grow(c, P.xval, P.xvalCap, 9 * (size_t)X)) != CS_OK) return st;
            cs_prox_outside_kernel<<<nblk(B.N, 128), 128, 0, c->stream>>>(B, P.rowPtr, P.rowInst, P.inst, P.xptr,
                                                                           P.xcol);
            CS_CUDA(cudaMemsetAsync(P.xval, 0, 9 * (size_t)X * sizeof(float), c->stream));
        }
        CS_CUDA(cudaGetLastError());
        CS_CUDA(cudaMemcpyAsync(touched.data(), P.sheetProx, B.S * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CS_CUDA(cudaStreamSynchronize(c->stream));
        B.n_pinst = T;
        B.pinst = P.inst;
        B.prec = P.rec;
        B.prow_ptr = P.rowPtr;
        B.prow_inst = P.rowInst;
        B.n_px = X;
        B.xptr = X > 0 ? P.xptr : nullptr;
        B.xcol = X > 0 ? P.xcol : nullptr;
        B.xval = X > 0 ? P.xval : nullptr;
        B.sheet_prox = P.sheetProx;
        P.n = n;
    }
    // sheets with proximities leave the cluster-resident kernel's work list for the batched
    // loop (their systems carry blocks outside the pattern, which only its SpMV reads)
    std::vector<int> rl;
    for (int s : c->rlistAll)
        if (!touched[s]) rl.push_back(s);
    if (!rl.empty()) CS_CUDA(cudaMemcpy(B.rlist, rl.data(), rl.size() * sizeof(int), cudaMemcpyHostToDevice));
    B.n_resident = (int)rl.size();
    c->rlistCur = rl;
    c->resClusters = std::min(c->resClustersMax, B.n_resident);
    return CS_OK;
}

// Host proximities: validated, copied to the device, applied.
cs_status setProximities(cs_ctx* c, const cs_proximity_desc* px, int n, float thickness) {
    if (n < 0 || (n > 0 && !px)) return fail(c, CS_ERR_INVALID_ARG, "bad proximity list");
    if (n > 0 && !(std::isfinite(thickness) && thickness > 0.0f))
        return fail(c, CS_ERR_INVALID_ARG, "repulsion thickness must be positive");
    Batch& B = c->B;
    auto finite = [](const float* a, int k) {
        for (int i = 0; i < k; i++)
            if (!std::isfinite(a[i])) return false;
        return true;
    };
    for (int p = 0; p < n; p++) {
        const cs_proximity_desc& d = px[p];
        for (int i = 0; i < 4; i++) {
            if (d.nodes[i] < -1 || d.nodes[i] >= B.N)
                return fail(c, CS_ERR_INVALID_ARG, "proximity %d: node %d out of range", p, d.nodes[i]);
            if (d.nodes[i] < 0 && !(finite(d.x[i], 3) && finite(d.v[i], 3)))
                return fail(c, CS_ERR_INVALID_ARG, "proximity %d: non-finite outside point", p);
            if (d.nodes[i] < 0 && ((d.free_mask >> i) & 1) && !(std::isfinite(d.mass[i]) && d.mass[i] > 0.0f))
                return fail(c, CS_ERR_INVALID_ARG, "proximity %d: free outside point without a positive mass", p);
        }
        if (!finite(d.normal, 3) || !finite(d.w, 4) || !std::isfinite(d.mu) || !std::isfinite(d.stiffness))
            return fail(c, CS_ERR_INVALID_ARG, "proximity %d: non-finite normal, weights or coefficients", p);
    }
    CS_CUDA(cudaSetDevice(c->device));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    cs_status st;
    if (n > 0) {
        if ((st = grow(c, c->prox.desc, c->prox.descCap, (size_t)n)) != CS_OK) return st;
        CS_CUDA(cudaMemcpyAsync(c->prox.desc, px, n * sizeof(cs_proximity_desc), cudaMemcpyHostToDevice, c->stream));
    }
    return applyProximities(c, n, thickness);
}

template <class T>
cs_status contactAlloc(cs_ctx* c, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return fail(c, CS_ERR_CUDA, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
    c->contactAllocs.push_back(q);
    *p = (T*)q;
    return CS_OK;
}

// Scene-wide edges, face edges, node-face adjacency and rest areas for detection (once per batch).
cs_status buildContact(cs_ctx* c) {
    Batch& B = c->B;
    Contact& C = c->contact;
    std::vector<float> farea(B.F);
    CS_CUDA(cudaMemcpy(farea.data(), B.face_area, B.F * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<int4> fedges, edges;
    std::vector<int> nfptr{0}, nfcode;
    std::vector<float> narea(B.N, 0.0f), earea;
    int eoff = 0;
    for (int s = 0; s < B.S; s++) {
        const Topo& T = *c->sheetTopo[s];
        const SheetDesc& sd = c->sheets[s];
        const int noff = sd.node_off, foff = sd.face_off;
        for (int f = 0; f < T.n_faces; f++)
            fedges.push_back(make_int4(eoff + T.f_edges[3 * f], eoff + T.f_edges[3 * f + 1], eoff + T.f_edges[3 * f + 2], s));
        const int ne = (int)T.e_nodes.size() / 2;
        for (int e = 0; e < ne; e++) {
            const int f0 = T.e_faces[2 * e], f1 = T.e_faces[2 * e + 1];
            edges.push_back(make_int4(noff + T.e_nodes[2 * e], noff + T.e_nodes[2 * e + 1], f0 < 0 ? -1 : foff + f0,
                                      f1 < 0 ? -1 : foff + f1));
            // Edge::area (Edge.cu:89-95)
            float a = 0.0f;
            if (f0 >= 0) a += farea[foff + f0];
            if (f1 >= 0) a += farea[foff + f1];
            earea.push_back(a);
        }
        for (int i = 0; i < T.n_nodes; i++) {
            for (int k = T.nf_ptr[i]; k < T.nf_ptr[i + 1]; k++) nfcode.push_back(T.nf_code[k] + (foff << 2));
            nfptr.push_back((int)nfcode.size());
        }
        // Mesh::updateNodeGeometries (Mesh.cu:190-198): a third of each face's area, faces in order
        for (int f = 0; f < T.n_faces; f++) {
            const float a = farea[foff + f] / 3.0f;
            for (int k = 0; k < 3; k++) narea[noff + T.fx[3 * f + k]] += a;
        }
        eoff += ne;
    }
    C.E = eoff;
    C.n_keys = (int)std::min<long long>(2LL * (B.N + (long long)C.E + B.F), INT32_MAX);
    if (2LL * (B.N + (long long)C.E + B.F) >= INT32_MAX || (long long)B.F * 8 >= INT32_MAX)
        return fail(c, CS_ERR_INVALID_ARG, "batch too large for proximity detection");
    int bits = 10;
    while ((1LL << bits) < 4LL * B.F && bits < 30) bits++;
    C.hash_bits = bits;
    cs_status st;
    int4 *dfe = nullptr, *de = nullptr;
    int *dnp = nullptr, *dnc = nullptr;
    float *dna = nullptr, *dea = nullptr;
#define CUP(ptr, vec)                                                                                    \
    if ((st = contactAlloc(c, &ptr, vec.size())) != CS_OK) return st;                                    \
    if (!vec.empty()) CS_CUDA(cudaMemcpy(ptr, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice));
    CUP(dfe, fedges);
    CUP(de, edges);
    CUP(dnp, nfptr);
    CUP(dnc, nfcode);
    CUP(dna, narea);
    CUP(dea, earea);
#undef CUP
    C.face_edges = dfe;
    C.edges = de;
    C.nf_ptr = dnp;
    C.nf_code = dnc;
    C.node_area = dna;
    C.edge_area = dea;
#define CAL(ptr, n) \
    if ((st = contactAlloc(c, &ptr, (size_t)(n))) != CS_OK) return st;
    CAL(C.fn, 3LL * B.F);
    CAL(C.nn, 3LL * B.N);
    CAL(C.box, 6LL * B.F);
    CAL(C.ext, 2);
    CAL(C.head, 1LL << bits);
    CAL(C.next, 8LL * B.F);
    CAL(C.keys, (long long)C.n_keys);
    CAL(C.block_count, (C.n_keys + CS_CONTACT_ITEMS - 1) / CS_CONTACT_ITEMS);
    CAL(C.total, 1);
    CAL(C.pair_count, 1);
    CAL(c->sheetGroupDev, B.S);
#undef CAL
    c->contactReady = true;
    return CS_OK;
}

// Candidate face pairs of the contact grid (contact.cu) with the dilation and bounds mode set
// in c->contact: face bounds (and, for proximities, node normals), the grid, the pairs
// (buffer regrown and the pass repeated when it was too small).
cs_status candidatePairs(cs_ctx* c, const int* sheetGroup, int& npairs) {
    Batch& B = c->B;
    Contact& C = c->contact;
    cs_status st;
    std::vector<int> groups(B.S, 0);
    if (sheetGroup) groups.assign(sheetGroup, sheetGroup + B.S);
    CS_CUDA(cudaMemcpyAsync(c->sheetGroupDev, groups.data(), B.S * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CS_CUDA(cudaMemsetAsync(C.ext, 0, 2 * sizeof(unsigned), c->stream));
    CS_CUDA(cudaMemsetAsync(C.head, 0xFF, (sizeof(int) << C.hash_bits), c->stream));
    cs_contact_face_kernel<<<nblk(B.F, 128), 128, 0, c->stream>>>(B, C);
    if (!C.ccd) cs_contact_node_kernel<<<nblk(B.N, 128), 128, 0, c->stream>>>(B, C);
    cs_contact_grid_kernel<<<nblk(B.F, 128), 128, 0, c->stream>>>(B, C, c->sheetGroupDev);
    npairs = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        if (C.pair_cap == 0 || npairs > C.pair_cap) {
            size_t cap = (size_t)C.pair_cap;
            if ((st = grow(c, C.pairs, cap, std::max<size_t>((size_t)npairs, 8 * (size_t)B.F))) != CS_OK) return st;
            C.pair_cap = (int)std::min<size_t>(cap, INT32_MAX);
        }
        CS_CUDA(cudaMemsetAsync(C.pair_count, 0, sizeof(int), c->stream));
        cs_contact_pair_kernel<<<nblk(B.F, 128), 128, 0, c->stream>>>(B, C, c->sheetGroupDev);
        CS_CUDA(cudaMemcpyAsync(&npairs, C.pair_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CS_CUDA(cudaStreamSynchronize(c->stream));
        if (npairs <= C.pair_cap) break;
    }
    CS_CUDA(cudaGetLastError());
    unsigned flags[2];
    CS_CUDA(cudaMemcpy(flags, C.ext, sizeof(flags), cudaMemcpyDeviceToHost));
    if (flags[1] & 1u) return fail(c, CS_ERR_INVALID_ARG, "non-finite node state");
    if (flags[1]) return fail(c, CS_ERR_STATE, "contact grid overflow (flags %u)", flags[1]);
    if (npairs > C.pair_cap) return fail(c, CS_ERR_STATE, "candidate pair buffer overflow");
    return CS_OK;
}

// Scratch of the collision step: node-sized arrays once per batch, impact-sized ones grown.
// The found impacts [0, n) into K.sorted by (time, node ids, type, index): four stable radix
// sorts over the key parts, least significant first (cs_impact_keys_kernel), then one gather;
// *pin = the permutation buffer holding the order.
cs_status sortImpacts(cs_ctx* c, int nFound, int* pin_out) {
    Collide& K = c->coll;
    int pin = 0;
    for (int pass = 0; pass < 4; pass++) {
        cs_impact_keys_kernel<<<nblk(nFound, 256), 256, 0, c->stream>>>(K, nFound, pass, K.sperm[pin], K.skey[0],
                                                                       K.sperm[pin]);
        size_t bytes = K.stmp_bytes;
        CS_CUDA(cub::DeviceRadixSort::SortPairs(K.stmp, bytes, K.skey[0], K.skey[1], K.sperm[pin], K.sperm[pin ^ 1],
                                                nFound, 0, pass == 0 ? 1 : pass == 2 ? 32 : 64, c->stream));
        pin ^= 1;
    }
    cs_impact_gather_kernel<<<nblk(nFound, 256), 256, 0, c->stream>>>(K, nFound, K.sperm[pin]);
    *pin_out = pin;
    return CS_OK;
}

cs_status collideScratch(cs_ctx* c, int nFound, int nAll) {
    Batch& B = c->B;
    Collide& K = c->coll;
    CollideCaps& P = c->collCaps;
    cs_status st;
    if (!K.mark) {
        // per node (the projection's nodes are a subset of the batch's)
        const size_t N = (size_t)B.N;
        size_t cap = 0;
        auto once = [&](auto*& q, size_t n) {
            cap = 0;
            return grow(c, q, cap, n);
        };
        if ((st = once(K.mark, N + 1)) != CS_OK || (st = once(K.used, N)) != CS_OK ||
            (st = once(K.nodes, N)) != CS_OK || (st = once(K.nptr, N + 1)) != CS_OK ||
            (st = once(K.nfill, N + 1)) != CS_OK || (st = once(K.x1, 3 * N)) != CS_OK ||
            (st = once(K.cur, 3 * N)) != CS_OK || (st = once(K.next, 3 * N)) != CS_OK ||
            (st = once(K.grad, 3 * N)) != CS_OK || (st = once(K.nterm, N)) != CS_OK ||
            (st = once(K.gterm, N)) != CS_OK || (st = once(K.counters, 2)) != CS_OK ||
            (st = once(K.nodemin, N)) != CS_OK)
            return st;
        CS_CUDA(cudaMemset(K.used, 0, N * sizeof(int)));
    }
    if ((size_t)nFound > P.found) {
        if ((st = grow(c, K.found, P.found, (size_t)nFound)) != CS_OK) return st;
        size_t cap = 0;
        if (K.sorted) cudaFree(K.sorted);
        K.sorted = nullptr;
        if ((st = grow(c, K.sorted, cap, P.found)) != CS_OK) return st;
        for (int** q : {&K.alive, &K.chosen, &K.sperm[0], &K.sperm[1]}) {
            if (*q) cudaFree(*q);
            *q = nullptr;
            cap = 0;
            if ((st = grow(c, *q, cap, P.found + 1)) != CS_OK) return st;
        }
        for (unsigned long long** q : {&K.skey[0], &K.skey[1]}) {
            if (*q) cudaFree(*q);
            *q = nullptr;
            cap = 0;
            if ((st = grow(c, *q, cap, P.found)) != CS_OK) return st;
        }
        // temp storage of the radix sorts (impactSort), for the largest key width
        size_t bytes = 0;
        for (int bits : {1, 32, 64}) {
            size_t b = 0;
            CS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, K.skey[0], K.skey[1], K.sperm[0], K.sperm[1],
                                                    (int)std::min<size_t>(P.found, INT32_MAX), 0, bits, c->stream));
            bytes = std::max(bytes, b);
        }
        if (K.stmp) cudaFree(K.stmp);
        K.stmp = nullptr;
        K.stmp_bytes = 0;
        CS_CUDA(cudaMalloc(&K.stmp, std::max<size_t>(bytes, 16)));
        K.stmp_bytes = std::max<size_t>(bytes, 16);
        K.found_cap = (int)std::min<size_t>(P.found, INT32_MAX);
    }
    if ((size_t)nAll > P.all) {
        // the accumulated impacts survive a regrow
        ImpactRec* old = K.all;
        const size_t oldCap = P.all;
        K.all = nullptr;
        P.all = 0;
        if ((st = grow(c, K.all, P.all, (size_t)nAll)) != CS_OK) return st;
        if (old) {
            CS_CUDA(cudaMemcpyAsync(K.all, old, oldCap * sizeof(ImpactRec), cudaMemcpyDeviceToDevice, c->stream));
            CS_CUDA(cudaStreamSynchronize(c->stream));
            cudaFree(old);
        }
        // per constraint (reallocated: their contents are rebuilt each round)
        auto fresh = [&](auto*& q, size_t n) {
            if (q) cudaFree(q);
            q = nullptr;
            size_t cap = 0;
            return grow(c, q, cap, n);
        };
        if ((st = fresh(K.idx, 4 * P.all)) != CS_OK || (st = fresh(K.nlist, 4 * P.all)) != CS_OK ||
            (st = fresh(K.lambda, P.all)) != CS_OK || (st = fresh(K.coef, P.all)) != CS_OK ||
            (st = fresh(K.cterm, P.all)) != CS_OK)
            return st;
    }
    return CS_OK;
}

}  // namespace

extern "C" {

cs_status cs_set_proximities(cs_ctx* c, const cs_proximity_desc* px, int n, float thickness) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    return setProximities(c, px, n, thickness);
}

// Simulator::physicsStep's detection (Simulator.cu:571-586, findProximitiesGpu :300-349) on
// the batch's current state, then cs_set_proximities with the result.
cs_status cs_detect_proximities(cs_ctx* c, const cs_detect_params* p, int* count) {
    if (!c || !p) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    if (!(std::isfinite(p->repulsion_thickness) && p->repulsion_thickness > 0.0f) || !std::isfinite(p->collision_stiffness) ||
        !std::isfinite(p->friction))
        return fail(c, CS_ERR_INVALID_ARG, "detection parameters must be finite, the thickness positive");
    CS_CUDA(cudaSetDevice(c->device));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    cs_status st;
    if (!c->contactReady && (st = buildContact(c)) != CS_OK) return st;
    Batch& B = c->B;
    Contact& C = c->contact;
    C.repulsion = p->repulsion_thickness;
    C.stiffness = p->collision_stiffness;
    C.friction = p->friction;
    C.dilate = 2.0f * p->repulsion_thickness;  // Simulator.cu:274
    C.ccd = 0;
    int npairs = 0;
    if ((st = candidatePairs(c, p->sheet_group, npairs)) != CS_OK) return st;
    CS_CUDA(cudaMemsetAsync(C.keys, 0xFF, (size_t)C.n_keys * sizeof(unsigned long long), c->stream));
    const int nblocks = (C.n_keys + CS_CONTACT_ITEMS - 1) / CS_CONTACT_ITEMS;
    if (npairs > 0) {
        cs_contact_vf_kernel<<<nblk(6LL * npairs, 256), 256, 0, c->stream>>>(B, C, npairs);
        cs_contact_ee_kernel<<<nblk(9LL * npairs, 256), 256, 0, c->stream>>>(B, C, npairs);
    }
    cs_contact_count_kernel<<<nblocks, 256, 0, c->stream>>>(C);
    cs_contact_scan_kernel<<<1, 1024, 0, c->stream>>>(C, nblocks);
    CS_CUDA(cudaGetLastError());
    int total = 0;
    CS_CUDA(cudaMemcpyAsync(&total, C.total, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    if ((st = grow(c, c->prox.desc, c->prox.descCap, (size_t)std::max(total, 1))) != CS_OK) return st;
    C.out = c->prox.desc;
    C.out_cap = (int)std::min<size_t>(c->prox.descCap, INT32_MAX);
    cs_contact_write_kernel<<<nblocks, 256, 0, c->stream>>>(B, C);
    CS_CUDA(cudaGetLastError());
    if ((st = applyProximities(c, total, p->repulsion_thickness)) != CS_OK) return st;
    if (count) *count = total;
    return CS_OK;
}

// Simulator::collisionStep (Simulator.cu:602-684, its GPU branch) after cs_step: rounds of
// continuous impact detection between x0 and x, selection of independent impacts and
// projection of all impacts found so far (collide.cu), up to 100 rounds on each of the two
// deformation levels; then v = (x - x0) / dt for every node.
cs_status cs_collision_step(cs_ctx* c, const cs_collision_params* p, cs_collision_stats* out) {
    if (!c || !p) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    if (!(std::isfinite(p->thickness) && p->thickness > 0.0f) || !(std::isfinite(p->dt) && p->dt > 0.0f))
        return fail(c, CS_ERR_INVALID_ARG, "collision thickness and time step must be positive");
    CS_CUDA(cudaSetDevice(c->device));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    cs_status st;
    if (!c->contactReady && (st = buildContact(c)) != CS_OK) return st;
    Batch& B = c->B;
    Contact& C = c->contact;
    Collide& K = c->coll;
    if ((st = collideScratch(c, 1, 1)) != CS_OK) return st;
    K.thickness = p->thickness;
    C.dilate = p->thickness;  // traverse with the collision thickness (Simulator.cu:385)
    C.ccd = 1;
    CS_CUDA(cudaMemcpyAsync(K.x1, B.x, 3 * (size_t)B.N * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
    int rounds = 0, total = 0;
    bool success = false;
    for (int deform = 0; deform < 2 && !success; deform++) {
        int nAll = 0;
        for (int round = 0; round < 100; round++) {
            rounds++;
            int npairs = 0;
            st = candidatePairs(c, p->sheet_group, npairs);
            if (st != CS_OK) {
                C.ccd = 0;
                return st;
            }
            int nFound = 0;
            for (int attempt = 0; attempt < 2; attempt++) {
                if ((st = collideScratch(c, std::max(nFound, 1024), nAll + 1)) != CS_OK) return st;
                CS_CUDA(cudaMemsetAsync(K.counters, 0, 2 * sizeof(int), c->stream));
                if (npairs > 0) {
                    // 256 threads, 2,048 (pair, test) items per block (collide.cu)
                    cs_impact_kernel<<<nblk(15LL * npairs, 2048), 256, 0, c->stream>>>(B, C, K, npairs);
                }
                CS_CUDA(cudaMemcpyAsync(&nFound, K.counters, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
                CS_CUDA(cudaStreamSynchronize(c->stream));
                if (nFound <= K.found_cap) break;
            }
            if (nFound == 0) {
                success = true;
                break;
            }
            if (nFound > K.found_cap) return fail(c, CS_ERR_STATE, "impact buffer overflow");
            if ((st = collideScratch(c, nFound, nAll + nFound)) != CS_OK) return st;
            // the round's impacts in order (time, node ids, type, index)
            int pin = 0;
            if ((st = sortImpacts(c, nFound, &pin)) != CS_OK) return st;
            // independent impacts: rounds of per-node minima until no impact is live
            const int g = nblk(nFound, 256);
            cs_select_init_kernel<<<nblk(nFound + 1, 256), 256, 0, c->stream>>>(K, nFound);
            for (int pass = 0; pass < nFound; pass++) {
                int live = 0;
                cs_select_reset_kernel<<<g, 256, 0, c->stream>>>(K, nFound);
                cs_select_min_kernel<<<g, 256, 0, c->stream>>>(K, nFound);
                cs_select_choose_kernel<<<g, 256, 0, c->stream>>>(K, nFound);
                CS_CUDA(cudaMemsetAsync(K.counters + 1, 0, sizeof(int), c->stream));
                cs_select_drop_kernel<<<g, 256, 0, c->stream>>>(K, nFound);
                CS_CUDA(cudaMemcpyAsync(&live, K.counters + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
                CS_CUDA(cudaStreamSynchronize(c->stream));
                if (live == 0) break;
            }
            int sel = 0;
            if ((st = scanInts(c, K.chosen, nFound, &sel)) != CS_OK) return st;
            cs_select_write_kernel<<<g, 256, 0, c->stream>>>(K, nFound, nAll, (int)c->collCaps.all);
            nAll += sel;
            total += sel;
            // the projection's nodes and constraints
            CS_CUDA(cudaMemsetAsync(K.mark, 0, ((size_t)B.N + 1) * sizeof(int), c->stream));
            cs_opt_mark_kernel<<<nblk(4LL * nAll, 256), 256, 0, c->stream>>>(K, nAll);
            int nn = 0;
            if ((st = scanInts(c, K.mark, B.N, &nn)) != CS_OK) return st;
            cs_opt_nodes_kernel<<<nblk(B.N, 256), 256, 0, c->stream>>>(K, B.N);
            CS_CUDA(cudaMemsetAsync(K.nptr, 0, ((size_t)nn + 1) * sizeof(int), c->stream));
            CS_CUDA(cudaMemsetAsync(K.nfill, 0, ((size_t)nn + 1) * sizeof(int), c->stream));
            cs_opt_idx_kernel<<<nblk(4LL * nAll, 256), 256, 0, c->stream>>>(K, nAll);
            if ((st = scanInts(c, K.nptr, nn, nullptr)) != CS_OK) return st;
            cs_opt_fill_kernel<<<nblk(4LL * nAll, 256), 256, 0, c->stream>>>(K, nAll);
            cs_opt_sort_kernel<<<nblk(nn, 256), 256, 0, c->stream>>>(K, nn);
            cs_opt_kernel<<<1, 1024, 0, c->stream>>>(B, K, nn, nAll);
            CS_CUDA(cudaGetLastError());
        }
    }
    C.ccd = 0;
    cs_collide_velocity_kernel<<<nblk(3LL * B.N, 256), 256, 0, c->stream>>>(B, 1.0f / p->dt);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    if (out) {
        out->rounds = rounds;
        out->impacts = total;
    }
    if (!success) return fail(c, CS_ERR_NOT_CONVERGED, "collision step failed: impacts remain after %d rounds", rounds);
    return CS_OK;
}

cs_status cs_get_proximities(cs_ctx* c, cs_proximity_desc* out, int cap, int* count) {
    if (!c || (cap > 0 && !out)) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    const int n = c->prox.n;
    if (n > 0 && cap > 0) {
        CS_CUDA(cudaStreamSynchronize(c->stream));
        CS_CUDA(cudaMemcpy(out, c->prox.desc, std::min(n, cap) * sizeof(cs_proximity_desc), cudaMemcpyDeviceToHost));
    }
    if (count) *count = n;
    return CS_OK;
}

cs_status cs_get_state(cs_ctx* c, float* x, float* v) {
    if (!c || (!x && !v)) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    size_t n = 3 * (size_t)c->B.N * sizeof(float);
    if (x) CS_CUDA(cudaMemcpyAsync(x, c->B.x, n, cudaMemcpyDeviceToHost, c->stream));
    if (v) CS_CUDA(cudaMemcpyAsync(v, c->B.v, n, cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

cs_status cs_set_state_device(cs_ctx* c, const float* x, const float* v) {
    if (!c || (!x && !v)) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    size_t n = 3 * (size_t)c->B.N * sizeof(float);
    if (x) CS_CUDA(cudaMemcpyAsync(c->B.x, x, n, cudaMemcpyDeviceToDevice, c->stream));
    if (v) CS_CUDA(cudaMemcpyAsync(c->B.v, v, n, cudaMemcpyDeviceToDevice, c->stream));
    return CS_OK;
}

cs_status cs_get_state_device(cs_ctx* c, float* x, float* v) {
    if (!c || (!x && !v)) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    size_t n = 3 * (size_t)c->B.N * sizeof(float);
    if (x) CS_CUDA(cudaMemcpyAsync(x, c->B.x, n, cudaMemcpyDeviceToDevice, c->stream));
    if (v) CS_CUDA(cudaMemcpyAsync(v, c->B.v, n, cudaMemcpyDeviceToDevice, c->stream));
    return CS_OK;
}

cs_status cs_device_pointers(cs_ctx* c, float** x, float** v, float** dv) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    if (x) *x = c->B.x;
    if (v) *v = c->B.v;
    if (dv) *dv = c->B.dv;
    return CS_OK;
}

static cs_status validateParams(cs_ctx* c, const cs_step_params* p) {
    if (!p) return fail(c, CS_ERR_INVALID_ARG, "null params");
    if (!(p->dt > 0.0f) || !std::isfinite(p->dt)) return fail(c, CS_ERR_INVALID_ARG, "dt must be positive");
    if (!std::isfinite(p->handle_stiffness) || p->handle_stiffness < 0) return fail(c, CS_ERR_INVALID_ARG, "bad handle stiffness");
    for (int i = 0; i < 3; i++)
        if (!std::isfinite(p->gravity[i])) return fail(c, CS_ERR_INVALID_ARG, "bad gravity");
    if (p->precision != CS_PREC_PLAIN_FP32 && p->precision != CS_PREC_MIXED) return fail(c, CS_ERR_INVALID_ARG, "bad precision");
    if (p->warm_start < CS_WARM_ZERO || p->warm_start > CS_WARM_GIVEN) return fail(c, CS_ERR_INVALID_ARG, "bad warm start");
    if (p->solver != CS_SOLVER_AUTO && p->solver != CS_SOLVER_BATCHED) return fail(c, CS_ERR_INVALID_ARG, "bad solver");
    if (p->precond_degree < 0 || p->precond_degree > CS_PRECOND_MAX_DEGREE || (p->precond_degree > 1 && p->precond_degree % 2 == 0))
        return fail(c, CS_ERR_INVALID_ARG, "precond_degree must be 0, 1 or odd up to CS_PRECOND_MAX_DEGREE");
    if (p->warm_start == CS_WARM_LEARNED && !c->mlpInit)
        return fail(c, CS_ERR_NOT_TRAINED, "learned warm start: no network (cs_mlp_init / cs_mlp_set_weights)");
    const int nt = p->transformations ? p->n_transformations : 0;
    if (nt < 0 || nt > CS_MAX_MOTIONS) return fail(c, CS_ERR_INVALID_ARG, "n_transformations must be 0..%d", CS_MAX_MOTIONS);
    if (nt > 0 && !p->transformations) return fail(c, CS_ERR_INVALID_ARG, "null transformations");
    for (int k = 0; k < nt * CS_TRANSFORM_FLOATS; k++)
        if (!std::isfinite(p->transformations[k])) return fail(c, CS_ERR_INVALID_ARG, "non-finite transformation");
    if (c->maxHandleMotion >= nt)
        return fail(c, CS_ERR_INVALID_ARG, "a handle follows motion %d but the step has %d transformations",
                    c->maxHandleMotion, nt);
    return CS_OK;
}

cs_status cs_set_handle_motions(cs_ctx* c, const int32_t* motion, int n) {
    if (!c || (n > 0 && !motion)) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    if (n != (int)c->handleNode.size())
        return fail(c, CS_ERR_INVALID_ARG, "%d motions given for %d handles", n, (int)c->handleNode.size());
    std::vector<int> per(c->B.N, -1);
    int mx = -1;
    for (int h = 0; h < n; h++) {
        if (motion[h] < -1 || motion[h] >= CS_MAX_MOTIONS)
            return fail(c, CS_ERR_INVALID_ARG, "handle %d: motion %d out of range (-1..%d)", h, motion[h], CS_MAX_MOTIONS - 1);
        per[c->handleNode[h]] = motion[h];  // a node's last handle, as for its target (cs_load_batch)
        mx = std::max(mx, motion[h]);
    }
    CS_CUDA(cudaSetDevice(c->device));
    CS_CUDA(cudaMemcpyAsync(c->B.handle_motion, per.data(), per.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    c->maxHandleMotion = mx;
    return CS_OK;
}

cs_status cs_assemble(cs_ctx* c, const cs_step_params* p) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    cs_status st = validateParams(c, p);
    if (st != CS_OK) return st;
    CS_CUDA(cudaSetDevice(c->device));
    DevParams d = toDev(p);
    CS_CUDA(cudaMemcpyAsync(c->B.params, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream));
    launchAssembly(c);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

// The step statistics of the last solve (per-sheet states, trip count), and the status it
// implies; `timed`: the step's duration between the context's events.
static cs_status fillStepStats(cs_ctx* c, cs_step_stats* stats, int loop_cap, bool timed) {
    std::vector<InstState> inst(c->B.S);
    int loopv[8];
    CS_CUDA(cudaMemcpyAsync(inst.data(), c->B.inst, c->B.S * sizeof(InstState), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaMemcpyAsync(loopv, c->B.loop, sizeof(loopv), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    memset(stats, 0, sizeof(*stats));
    stats->n_instances = c->B.S;
    stats->loop_trips = loopv[0];
    bool capped = false, breakdown = false;
    for (int s = 0; s < c->B.S; s++) {
        const InstState& I = inst[s];
        stats->converged += (I.flags & CS_IF_CONVERGED) ? 1 : 0;
        stats->max_iters = std::max(stats->max_iters, I.iters);
        stats->total_iters += I.iters;
        stats->max_sweeps = std::max(stats->max_sweeps, I.sweeps);
        stats->warm_rejected += (I.flags & CS_IF_WARM_REJECTED) ? 1 : 0;
        double bn = std::sqrt(I.bnorm2);
        double rel = bn > 0 ? I.resnorm / bn : 0.0;
        stats->max_rel_residual = std::max(stats->max_rel_residual, rel);
        if (!(I.flags & CS_IF_CONVERGED)) capped = true;
        if (I.flags & CS_IF_BREAKDOWN) breakdown = true;
    }
    float ms = 0.f;
    if (timed) CS_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    stats->ms = ms;
    if (loopv[0] >= loop_cap) return fail(c, CS_ERR_TIMEOUT, "solve loop hit its trip bound (%d)", loop_cap);
    if (loopv[6]) return fail(c, CS_ERR_TIMEOUT, "cluster-resident solve: a wait on another CTA ran out");
    if (capped) return fail(c, breakdown ? CS_ERR_NON_SPD : CS_ERR_NOT_CONVERGED, "%d of %d sheets did not converge",
                            c->B.S - stats->converged, c->B.S);
    return CS_OK;
}

cs_status cs_step(cs_ctx* c, const cs_step_params* p, cs_step_stats* stats) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    cs_status st = validateParams(c, p);
    if (st != CS_OK) return st;
    CS_CUDA(cudaSetDevice(c->device));
    DevParams d = toDev(p);
    c->hostParams = d;
    CS_CUDA(cudaMemcpyAsync(c->B.params, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream));
    if ((st = setTripCoarse(c, p->coarse != 0)) != CS_OK) return st;
    CS_CUDA(cudaEventRecord(c->ev0, c->stream));
    const bool learned = p->warm_start == CS_WARM_LEARNED;
    if (p->use_graph) {
        if ((st = buildGraph(c, learned)) != CS_OK) return st;
        CS_CUDA(cudaGraphLaunch(c->gexec[learned][c->tripCoarse], c->stream));
    } else {
        c->hostLaunches += assemblyKernels(c) + 3 + bcSetupKernels(c) + residentKernels(c) + (learned ? 3 : 0);
        launchPrelude(c, learned);
        int go = 1;
        int trips = 0;
        while (go) {
            for (int t = 0; t < 8; t++) launchTrip(c, 0);
            trips += 8;
            CS_CUDA(cudaMemcpyAsync(&go, c->B.loop + 3, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
            CS_CUDA(cudaStreamSynchronize(c->stream));
            if (trips > d.loop_cap + 16) break;
        }
        cs_advance_kernel<<<nblk(3LL * c->B.N, 256), 256, 0, c->stream>>>(c->B);
    }
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaEventRecord(c->ev1, c->stream));
    c->lastStepValid = true;
    c->steps++;
    if (p->use_graph) {
        c->graphSteps++;
        c->graphLaunchesFixed += assemblyKernels(c) + 3 + (learned ? 3 : 0) + bcSetupKernels(c) + residentKernels(c);
    }
    if (!stats) return CS_OK;
    return fillStepStats(c, stats, d.loop_cap, true);
}

cs_status cs_sync(cs_ctx* c) {
    if (!c) return CS_ERR_INVALID_ARG;
    CS_CUDA(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

cs_status cs_set_warm_start(cs_ctx* c, const float* dv) {
    if (!c || !dv) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    CS_CUDA(cudaMemcpyAsync(c->B.warm, dv, 3 * (size_t)c->B.N * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    return CS_OK;
}

cs_status cs_get_dv(cs_ctx* c, float* dv) {
    if (!c || !dv) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    CS_CUDA(cudaMemcpyAsync(dv, c->B.dv, 3 * (size_t)c->B.N * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

cs_status cs_get_instance_stats(cs_ctx* c, int* iters, double* rel, int* flags) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->loaded || !c->lastStepValid) return fail(c, CS_ERR_STATE, "no step run");
    std::vector<InstState> inst(c->B.S);
    CS_CUDA(cudaMemcpyAsync(inst.data(), c->B.inst, c->B.S * sizeof(InstState), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    for (int s = 0; s < c->B.S; s++) {
        if (iters) iters[s] = inst[s].iters;
        double bn = std::sqrt(inst[s].bnorm2);
        if (rel) rel[s] = bn > 0 ? inst[s].resnorm / bn : 0.0;
        if (flags) flags[s] = inst[s].flags;
    }
    return CS_OK;
}

cs_status cs_get_system(cs_ctx* c, int32_t* row_ptr, int32_t* col, float* val, float* b) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    const Batch& B = c->B;
    std::vector<float> A((size_t)B.n_panels * CS_PANEL_FLOATS);
    CS_CUDA(cudaMemcpy(A.data(), B.A, A.size() * sizeof(float), cudaMemcpyDeviceToHost));
    if (b) CS_CUDA(cudaMemcpy(b, B.b, 3 * (size_t)B.N * sizeof(float), cudaMemcpyDeviceToHost));
    // proximity blocks outside the pattern, merged into each row in column order
    std::vector<float> X(9 * (size_t)B.n_px);
    std::vector<int> hxptr, hxcol(B.n_px);
    if (B.n_px > 0) {
        hxptr.resize((size_t)B.N + 1);
        CS_CUDA(cudaMemcpy(X.data(), B.xval, X.size() * sizeof(float), cudaMemcpyDeviceToHost));
        CS_CUDA(cudaMemcpy(hxptr.data(), B.xptr, hxptr.size() * sizeof(int), cudaMemcpyDeviceToHost));
        CS_CUDA(cudaMemcpy(hxcol.data(), B.xcol, hxcol.size() * sizeof(int), cudaMemcpyDeviceToHost));
    }
    long long pos = 0;
    int rowBase = 0;
    if (row_ptr) row_ptr[0] = 0;
    for (int s = 0; s < B.S; s++) {
        const Topo& T = *c->sheetTopo[s];
        const SheetDesc& sd = c->sheets[s];
        int panelBase = c->slices[sd.slice_off].panel0 - T.slice_tpanel0[0];
        for (int i = 0; i < T.n_nodes; i++) {
            const int row = rowBase + i;
            int m = B.n_px > 0 ? hxptr[row] : 0;
            const int mEnd = B.n_px > 0 ? hxptr[row + 1] : 0;
            auto putExtra = [&]() {
                if (col) col[pos] = hxcol[m];
                if (val) std::copy(X.begin() + 9 * (size_t)m, X.begin() + 9 * (size_t)m + 9, val + 9 * pos);
                pos++;
                m++;
            };
            for (int p = T.csr_ptr[i]; p < T.csr_ptr[i + 1]; p++) {
                while (m < mEnd && hxcol[m] < rowBase + T.csr_col[p]) putExtra();
                int slot = T.csr_slot[p];
                int lane = slot % CS_SLICE, panel = panelBase + slot / CS_SLICE;
                const float* P = A.data() + (size_t)panel * CS_PANEL_FLOATS;
                if (col) col[pos] = rowBase + T.csr_col[p];
                if (val) {
                    float* o = val + 9 * pos;
                    for (int t = 0; t < 4; t++) o[t] = P[4 * lane + t];
                    for (int t = 0; t < 4; t++) o[4 + t] = P[128 + 4 * lane + t];
                    o[8] = P[256 + lane];
                }
                pos++;
            }
            while (m < mEnd) putExtra();
            if (row_ptr) row_ptr[row + 1] = (int32_t)pos;
        }
        rowBase += T.n_nodes;
    }
    return CS_OK;
}

cs_status cs_get_element_forces(cs_ctx* c, float* face_f, float* face_J, float* edge_f, float* edge_J,
                                int32_t* edge_nodes) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    const Batch& B = c->B;
    float *dff = nullptr, *dfJ = nullptr, *def = nullptr, *deJ = nullptr;
    CS_CUDA(cudaMalloc(&dff, 9 * (size_t)B.F * sizeof(float)));
    CS_CUDA(cudaMalloc(&dfJ, 81 * (size_t)B.F * sizeof(float)));
    CS_CUDA(cudaMalloc(&def, 12 * (size_t)std::max(B.E, 1) * sizeof(float)));
    CS_CUDA(cudaMalloc(&deJ, 144 * (size_t)std::max(B.E, 1) * sizeof(float)));
    cs_expand_kernel<<<nblk(std::max(B.F, B.E), 128), 128, 0, c->stream>>>(B, dff, dfJ, def, deJ);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess && face_f) e = cudaMemcpy(face_f, dff, 9 * (size_t)B.F * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && face_J) e = cudaMemcpy(face_J, dfJ, 81 * (size_t)B.F * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && edge_f) e = cudaMemcpy(edge_f, def, 12 * (size_t)B.E * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && edge_J) e = cudaMemcpy(edge_J, deJ, 144 * (size_t)B.E * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && edge_nodes) e = cudaMemcpy(edge_nodes, B.edge_nodes, 16 * (size_t)B.E, cudaMemcpyDeviceToHost);
    cudaFree(dff);
    cudaFree(dfJ);
    cudaFree(def);
    cudaFree(deJ);
    if (e != cudaSuccess) return fail(c, CS_ERR_CUDA, "element force readback: %s", cudaGetErrorString(e));
    return CS_OK;
}

cs_status cs_spmv(cs_ctx* c, const float* x, float* y) {
    if (!c || !x || !y) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    size_t n = 3 * (size_t)c->B.N * sizeof(float);
    float *dx = nullptr, *dy = nullptr;
    CS_CUDA(cudaMalloc(&dx, n));
    CS_CUDA(cudaMalloc(&dy, n));
    cudaError_t e = cudaMemcpy(dx, x, n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        cs_spmv_plain_kernel<<<nblk((long long)c->B.n_slices * 32, 128), 128, 0, c->stream>>>(c->B, dx, dy);
        e = cudaStreamSynchronize(c->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, dy, n, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    if (e != cudaSuccess) return fail(c, CS_ERR_CUDA, "spmv: %s", cudaGetErrorString(e));
    return CS_OK;
}

cs_status cs_profile_kernels(cs_ctx* c, const cs_step_params* p, int reps, float* ms) {
    if (!c || !ms || reps <= 0) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    cs_status st = validateParams(c, p);
    if (st != CS_OK) return st;
    CS_CUDA(cudaSetDevice(c->device));
    Batch& B = c->B;
    DevParams d = toDev(p);
    CS_CUDA(cudaMemcpyAsync(B.params, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream));
    launchAssembly(c);
    const int g = nblk((long long)B.n_slices * 32, 128);
    auto timeIt = [&](int which) -> float {
        cudaEventRecord(c->ev0, c->stream);
        for (int r = 0; r < reps; r++) {
            switch (which) {
                case 1: if (B.E) cs_edge_kernel<<<nblk(B.E, 128), 128, 0, c->stream>>>(B); break;
                case 2: cs_gather_kernel<<<c->gatherGrid, 32 * c->gatherWarps, c->gatherSmem, c->stream>>>(B); break;
                case 3: launchSpmvShape(B, c->spmvShape, c->stream); break;
                case 4: cs_vector_kernel<<<g, 128, 0, c->stream>>>(B); break;
                case 5: cs_reduce1_kernel<<<B.S, CS_REDUCE_THREADS, 0, c->stream>>>(B); break;
                case 6: launchSpmvShape(B, c->spmvShape, c->stream); break;
            }
        }
        cudaEventRecord(c->ev1, c->stream);
        cudaEventSynchronize(c->ev1);
        float t = 0.f;
        cudaEventElapsedTime(&t, c->ev0, c->ev1);
        return t / reps;
    };
    // the face terms are evaluated inside the gather: entry 0 stays 0
    ms[0] = 0.f;
    ms[1] = timeIt(1);
    ms[2] = timeIt(2);
    // solver kernels with every instance held in one phase
    cs_solve_setup_kernel<<<B.S, 128, 0, c->stream>>>(B);
    cs_solve_prologue_kernel<<<nblk(3LL * B.N, 256), 256, 0, c->stream>>>(B);
    cs_profile_setup_kernel<<<nblk(B.S, 128), 128, 0, c->stream>>>(B, PH_CG);
    ms[3] = timeIt(3);
    ms[4] = timeIt(4);
    ms[5] = timeIt(5);
    cs_profile_setup_kernel<<<nblk(B.S, 128), 128, 0, c->stream>>>(B, PH_RES);
    ms[6] = timeIt(6);
    // the batched loop's coarse correction (coarse.cu): its per-step set-up for the sheets the
    // loop solves, and one trip's kernels (R r, A_c^-1 R r, z += R^T e_c with the partials)
    ms[9] = ms[10] = 0.f;
    if (B.bc_total_agg > 0 && p->coarse) {
        cs_slice_bnorm_kernel<<<nblk((long long)B.n_slices * 32, 128), 128, 0, c->stream>>>(B);
        cs_solve_setup_kernel<<<B.S, 128, 0, c->stream>>>(B);
        float t = 0.f;
        cudaEventRecord(c->ev0, c->stream);
        for (int r = 0; r < reps; r++) launchBatchedCoarseSetup(c);
        cudaEventRecord(c->ev1, c->stream);
        cudaEventSynchronize(c->ev1);
        cudaEventElapsedTime(&t, c->ev0, c->ev1);
        ms[9] = t / reps;
        cs_solve_prologue_kernel<<<nblk(3LL * B.N, 256), 256, 0, c->stream>>>(B);
        cudaEventRecord(c->ev0, c->stream);
        for (int r = 0; r < reps; r++) {
            cs_bc_restrict_kernel<<<B.bc_total_agg, 256, 0, c->stream>>>(B);
            cs_bc_apply_kernel<<<nblk((long long)B.bc_total_agg * 96, 256), 256, 0, c->stream>>>(B);
            cs_bc_finish_kernel<<<g, 128, 0, c->stream>>>(B);
        }
        cudaEventRecord(c->ev1, c->stream);
        cudaEventSynchronize(c->ev1);
        cudaEventElapsedTime(&t, c->ev0, c->ev1);
        ms[10] = t / reps;
    }
    // one whole cluster-resident solve of every resident sheet from the zero guess (or the
    // warm start the parameters ask for); set-up launches untimed, the solve between events
    ms[7] = ms[8] = 0.f;
    if (c->resClusters > 0) {
        float acc = 0.f, accSetup = 0.f;
        for (int r = 0; r < reps; r++) {
            launchSolvePrologueAgain(c);
            cudaEventRecord(c->ev0, c->stream);
            launchCoarseSetup(c);
            cudaEventRecord(c->ev1, c->stream);
            cudaEventSynchronize(c->ev1);
            float t = 0.f;
            cudaEventElapsedTime(&t, c->ev0, c->ev1);
            accSetup += t;
            cudaEventRecord(c->ev0, c->stream);
            launchResident(c, false);
            cudaEventRecord(c->ev1, c->stream);
            cudaEventSynchronize(c->ev1);
            cudaEventElapsedTime(&t, c->ev0, c->ev1);
            acc += t;
        }
        ms[7] = acc / reps;
        ms[8] = accSetup / reps;
    }

    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    // the per-sheet statistics of the last timed resident solve stay readable when it solved
    // every sheet of the batch
    c->lastStepValid = c->resClusters > 0 && c->B.n_resident == c->B.S;
    return CS_OK;
}

namespace {
// Order-independent checksum of 32-bit words (XOR of each word mixed with its index).
__global__ void cs_checksum_kernel(const uint32_t* __restrict__ w, long long n, unsigned salt, unsigned* out) {
    unsigned acc = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned h = w[i] ^ (unsigned)(i * 0x9E3779B1ull) ^ salt;
        h ^= h >> 16;
        h *= 0x85EBCA6Bu;
        h ^= h >> 13;
        acc ^= h;
    }
    atomicXor(out, acc);
}
}  // namespace

// One whole solve of the loaded system (already assembled) with parameters q, launched from
// the host (cluster-resident kernel, then the batched loop polled every 8 trips), timed with
// CUDA events on the context's stream; -1 if a launch failed.
static float timeWholeSolve(cs_ctx* c, const cs_step_params& q) {
    Batch& B = c->B;
    DevParams d = toDev(&q);
    if (setTripCoarse(c, q.coarse != 0) != CS_OK) return -1.f;
    if (cudaMemcpyAsync(B.params, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream) != cudaSuccess) return -1.f;
    launchSolvePrologueAgain(c);
    cudaEventRecord(c->ev0, c->stream);
    launchResident(c);
    int go = 1, trips = 0;
    while (go) {
        for (int t = 0; t < 8; t++) launchTrip(c, 0);
        trips += 8;
        if (cudaMemcpyAsync(&go, B.loop + 3, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            return -1.f;
        if (trips > d.loop_cap + 16) break;
    }
    cudaEventRecord(c->ev1, c->stream);
    if (cudaEventSynchronize(c->ev1) != cudaSuccess) return -1.f;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    return ms;
}

cs_status cs_tune(cs_ctx* c, const cs_step_params* p, int reps, cs_tune_result* out) {
    if (!c || reps <= 0) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    cs_status st = validateParams(c, p);
    if (st != CS_OK) return st;
    CS_CUDA(cudaSetDevice(c->device));
    Batch& B = c->B;
    DevParams d = toDev(p);
    CS_CUDA(cudaMemcpyAsync(B.params, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream));
    launchAssembly(c);
    // the SpMV's shapes on one fixed CG product (every instance in PH_CG, as cs_profile_kernels sets it)
    cs_solve_setup_kernel<<<B.S, 128, 0, c->stream>>>(B);
    cs_solve_prologue_kernel<<<nblk(3LL * B.N, 256), 256, 0, c->stream>>>(B);
    cs_profile_setup_kernel<<<nblk(B.S, 128), 128, 0, c->stream>>>(B, PH_CG);
    unsigned* sum = reinterpret_cast<unsigned*>(B.loop + 7);
    float bestMs = 1e30f;
    int best = c->spmvShape;
    for (int k = 0; k < CS_SPMV_CANDIDATES; k++) {
        CS_CUDA(cudaMemsetAsync(B.q, 0, 3LL * B.N * sizeof(float), c->stream));
        launchSpmvShape(B, k, c->stream);
        CS_CUDA(cudaMemsetAsync(sum, 0, sizeof(unsigned), c->stream));
        cs_checksum_kernel<<<256, 256, 0, c->stream>>>(reinterpret_cast<const uint32_t*>(B.q), 3LL * B.N, 1u, sum);
        cs_checksum_kernel<<<64, 256, 0, c->stream>>>(reinterpret_cast<const uint32_t*>(B.part), 4LL * B.n_slices, 2u, sum);
        unsigned h = 0;
        CS_CUDA(cudaMemcpyAsync(&h, sum, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        CS_CUDA(cudaEventRecord(c->ev0, c->stream));
        for (int r = 0; r < reps; r++) launchSpmvShape(B, k, c->stream);
        CS_CUDA(cudaEventRecord(c->ev1, c->stream));
        CS_CUDA(cudaEventSynchronize(c->ev1));
        float ms = 0.f;
        CS_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        ms /= reps;
        if (out) {
            out->spmv_ms[k] = ms;
            out->spmv_checksum[k] = h;
            out->spmv_threads[k] = kSpmvShapes[k].threads;
            out->spmv_spw[k] = kSpmvShapes[k].spw;
            out->spmv_unroll[k] = kSpmvShapes[k].unroll;
        }
        if (ms < bestMs) {
            bestMs = ms;
            best = k;
        }
    }
    c->spmvShape = best;
    if (out) out->best_spmv = best;
    // the resident solver's preconditioners: one whole solve of the resident sheets each
    static const int degs[CS_TUNE_PRECONDS] = {1, 3, 3, 5, 5, 7}, coarse[CS_TUNE_PRECONDS] = {0, 0, 1, 0, 1, 1};
    int bestP = -1;
    float bestPm = 1e30f;
    for (int k = 0; k < CS_TUNE_PRECONDS; k++) {
        float ms = 0.f;
        if (c->resClusters > 0) {
            cs_step_params q = *p;
            q.precond_degree = degs[k];
            q.coarse = coarse[k];
            q.solver = CS_SOLVER_AUTO;
            DevParams dq = toDev(&q);
            CS_CUDA(cudaMemcpyAsync(B.params, &dq, sizeof(dq), cudaMemcpyHostToDevice, c->stream));
            // one untimed solve, then the mean of up to three timed ones
            const int nrep = reps < 3 ? reps : 3;
            for (int r = 0; r <= nrep; r++) {
                launchSolvePrologueAgain(c);
                CS_CUDA(cudaEventRecord(c->ev0, c->stream));
                launchResident(c);
                CS_CUDA(cudaEventRecord(c->ev1, c->stream));
                CS_CUDA(cudaEventSynchronize(c->ev1));
                float t = 0.f;
                CS_CUDA(cudaEventElapsedTime(&t, c->ev0, c->ev1));
                if (r > 0) ms += t / nrep;
            }
            if (ms < bestPm) {
                bestPm = ms;
                bestP = k;
            }
        }
        if (out) {
            out->precond_ms[k] = ms;
            out->precond_degree[k] = degs[k];
            out->precond_coarse[k] = coarse[k];
        }
    }
    c->tunedDegree = bestP >= 0 ? degs[bestP] : 0;
    c->tunedCoarse = bestP >= 0 ? coarse[bestP] : 0;
    if (out) out->best_precond = bestP;
    // the whole solve by each route: resident sheets on the cluster kernel (with the fastest
    // preconditioner) and the rest in the batched loop, or every sheet in the batched loop
    // (which wins when sheets too large for a cluster set the loop's trip count anyway)
    {
        cs_step_params q = *p;
        if (bestP >= 0) {
            q.precond_degree = degs[bestP];
            q.coarse = coarse[bestP];
        }
        float ms[2] = {0.f, 0.f};
        for (int k = 0; k < 2; k++) {
            q.solver = k == 0 ? CS_SOLVER_AUTO : CS_SOLVER_BATCHED;
            if (k == 0 && c->resClusters <= 0) continue;
            const int nrep = reps < 2 ? reps : 2;
            for (int r = 0; r <= nrep; r++) {
                const float t = timeWholeSolve(c, q);
                if (t < 0.f) return fail(c, CS_ERR_CUDA, "cs_tune: solve timing failed");
                if (r > 0) ms[k] += t / nrep;
            }
        }
        const int bestS = (c->resClusters > 0 && ms[0] <= ms[1]) ? CS_SOLVER_AUTO : CS_SOLVER_BATCHED;
        c->tunedSolver = bestS;
        if (out) {
            out->solver_ms[0] = ms[0];
            out->solver_ms[1] = ms[1];
            out->best_solver = bestS;
        }
    }
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    destroyGraphs(c);  // the captured steps launch the old SpMV shape
    c->lastStepValid = false;
    return CS_OK;
}

cs_status cs_impact_order(cs_ctx* c, const int32_t* nodes, const float* t, const int32_t* type, int n,
                          int32_t* order) {
    if (!c || n < 0 || (n > 0 && (!nodes || !t || !type || !order))) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    if (n == 0) return CS_OK;
    for (int i = 0; i < n; i++) {
        if (!(t[i] >= 0.0f) || (type[i] != 0 && type[i] != 1))
            return fail(c, CS_ERR_INVALID_ARG, "impact %d: time below 0 or bad type", i);
        for (int k = 0; k < 4; k++)
            if (nodes[4 * i + k] < 0) return fail(c, CS_ERR_INVALID_ARG, "impact %d: negative node id", i);
    }
    CS_CUDA(cudaSetDevice(c->device));
    cs_status st = collideScratch(c, n, 1);
    if (st != CS_OK) return st;
    std::vector<ImpactRec> h(n);
    for (int i = 0; i < n; i++) {
        ImpactRec r{};
        for (int k = 0; k < 4; k++) r.nodes[k] = nodes[4 * i + k];
        r.t = t[i];
        r.type = type[i];
        h[i] = r;
    }
    Collide& K = c->coll;
    CS_CUDA(cudaMemcpyAsync(K.found, h.data(), n * sizeof(ImpactRec), cudaMemcpyHostToDevice, c->stream));
    int pin = 0;
    if ((st = sortImpacts(c, n, &pin)) != CS_OK) return st;
    CS_CUDA(cudaMemcpyAsync(order, K.sperm[pin], n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

cs_status cs_get_counters(cs_ctx* c, long long* out) {
    if (!c || !out) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    int loopv[8];
    CS_CUDA(cudaMemcpyAsync(loopv, c->B.loop, sizeof(loopv), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    long long trips = (long long)(unsigned)loopv[4];
    out[0] = c->steps;
    out[1] = trips;
    // graph steps: fixed kernels plus those of every loop trip; host-driven steps are counted directly
    out[2] = c->hostLaunches + c->graphLaunchesFixed + c->tripLaunchBase + tripKernels(c) * (trips - c->tripsBase);
    return CS_OK;
}

cs_status cs_get_stream(cs_ctx* c, void** stream) {
    if (!c || !stream) return CS_ERR_INVALID_ARG;
    *stream = (void*)c->stream;
    return CS_OK;
}

// ---------------------------------------------------------------------------------------
// Learned warm start (no reference counterpart; network in mlp.cu).

namespace {

uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

uint16_t to_bf16_bits(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

cs_status mlpUploadWeights(cs_ctx* c, const std::vector<float>& w) {
    std::vector<uint16_t> wb(MLP_P);
    for (int i = 0; i < MLP_P; i++) wb[i] = to_bf16_bits(w[i]);
    CS_CUDA(cudaMemcpy(c->mlp.w, w.data(), MLP_P * sizeof(float), cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemcpy(c->mlp.wb, wb.data(), MLP_P * 2, cudaMemcpyHostToDevice));
    CS_CUDA(cudaMemset(c->mlp.m, 0, MLP_P * sizeof(float)));
    CS_CUDA(cudaMemset(c->mlp.v, 0, MLP_P * sizeof(float)));
    c->adamStep = 0;
    return CS_OK;
}

cs_status mlpCheckErr(cs_ctx* c) {
    int e = 0;
    CS_CUDA(cudaMemcpy(&e, c->mlp.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(c, CS_ERR_TIMEOUT, "a tensor-core completion wait gave up");
    return CS_OK;
}

// One forward + backward pass over sheets [s0, s1) of dataset slot `slot`; leaves the
// per-CTA gradient partials and loss partials in place.
// Energy-norm forward and backward over sheets [s0, s1): features in M.feat, the system
// assembled, M.sheet_c holding each sheet's dv*^T b; the prediction goes to M.pred, its
// gradient partials to M.gpart and the sheets' losses to M.sheet_loss.
void mlpEnergyForwardBackward(cs_ctx* c, int s0, int s1) {
    Batch& B = c->B;
    MlpDev& M = c->mlp;
    const SheetDesc &a = c->sheets[s0], &z = c->sheets[s1 - 1];
    const int n0 = a.node_off, n1 = z.node_off + z.n_nodes;
    const int sl0 = a.slice_off, sl1 = z.slice_off + z.n_slices;
    cs_mlp_l1_kernel<<<c->mlpGridTile, 128, MLP_SMEM_L1, c->stream>>>(B, M, M.feat, n0, n1, M.z1);
    cs_mlp_l23_kernel<<<c->mlpGridTile, 128, MLP_SMEM_L23, c->stream>>>(B, M, n0, n1, M.z2, M.z3, M.y, M.pred);
    cs_mlp_energy_kernel<<<nblk((long long)(sl1 - sl0) * 32, 128), 128, 0, c->stream>>>(B, M, sl0, sl1);
    cs_mlp_energy_sheet_kernel<<<s1 - s0, 128, 0, c->stream>>>(B, M, s0, s1, 1);
    cs_mlp_bwd23_kernel<<<c->mlpGridTrain, 128, MLP_SMEM_BWD23, c->stream>>>(B, M, n0, n1, nullptr);
    cs_mlp_bwd1_kernel<<<c->mlpGridTrain, 128, MLP_SMEM_BWD1, c->stream>>>(B, M, M.feat, n0, n1);
}

// The first half of a training step: assembly for the current state, the features of that
// system (with the previous dv in B.warm), the solve (host-driven launches), and every sheet's
// solution energy dv*^T b.
cs_status mlpEnergyPrepare(cs_ctx* c, const cs_step_params* p) {
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    if (p->warm_start == CS_WARM_LEARNED)
        return fail(c, CS_ERR_INVALID_ARG, "training steps solve without the learned warm start");
    if (c->B.n_pinst > 0) return fail(c, CS_ERR_STATE, "training steps take batches without proximities");
    cs_status st = validateParams(c, p);
    if (st != CS_OK) return st;
    CS_CUDA(cudaSetDevice(c->device));
    Batch& B = c->B;
    MlpDev& M = c->mlp;
    DevParams d = toDev(p);
    if ((st = setTripCoarse(c, p->coarse != 0)) != CS_OK) return st;
    CS_CUDA(cudaMemcpyAsync(B.params, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream));
    launchAssembly(c);
    cs_mlp_features_kernel<<<nblk(B.N, 256), 256, 0, c->stream>>>(B, M, M.feat);
    launchSolvePrologue(c);
    launchResident(c);
    int go = 1, trips = 0;
    while (go) {
        for (int t = 0; t < 8; t++) launchTrip(c, 0);
        trips += 8;
        CS_CUDA(cudaMemcpyAsync(&go, B.loop + 3, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CS_CUDA(cudaStreamSynchronize(c->stream));
        if (trips > d.loop_cap + 16) break;
    }
    cs_mlp_energy_norm_kernel<<<nblk((long long)B.n_slices * 32, 128), 128, 0, c->stream>>>(B, M, 0, B.n_slices);
    cs_mlp_energy_sheet_kernel<<<B.S, 128, 0, c->stream>>>(B, M, 0, B.S, 0);
    CS_CUDA(cudaGetLastError());
    return CS_OK;
}

void mlpForwardBackward(cs_ctx* c, int slot, int s0, int s1) {
    Batch& B = c->B;
    MlpDev& M = c->mlp;
    const int n0 = c->sheets[s0].node_off;
    const int n1 = c->sheets[s1 - 1].node_off + c->sheets[s1 - 1].n_nodes;
    const float* f = M.dfeat + (size_t)slot * B.N * 16;
    const float* tg = M.dtarget + (size_t)slot * B.N * 3;
    cs_mlp_l1_kernel<<<c->mlpGridTile, 128, MLP_SMEM_L1, c->stream>>>(B, M, f, n0, n1, M.z1);
    cs_mlp_l23_kernel<<<c->mlpGridTile, 128, MLP_SMEM_L23, c->stream>>>(B, M, n0, n1, M.z2, M.z3, M.y, nullptr);
    cs_mlp_bwd23_kernel<<<c->mlpGridTrain, 128, MLP_SMEM_BWD23, c->stream>>>(B, M, n0, n1, tg);
    cs_mlp_bwd1_kernel<<<c->mlpGridTrain, 128, MLP_SMEM_BWD1, c->stream>>>(B, M, f, n0, n1);
}

}  // namespace

cs_status cs_mlp_init(cs_ctx* c, int slots, unsigned long long seed) {
    if (!c || slots < 0) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    if (c->mlpInit) return fail(c, CS_ERR_STATE, "network already initialised for this batch");
    CS_CUDA(cudaSetDevice(c->device));
    cudaDeviceProp prop;
    CS_CUDA(cudaGetDeviceProperties(&prop, c->device));
    c->mlpGridTile = 2 * prop.multiProcessorCount;
    // layer 1: 64 TMEM columns per CTA (8 per SM); layers 2-3: 128 columns and 51 KB of shared
    // memory per CTA (4 per SM: the SM's 512 TMEM columns)
    c->mlpGridL1 = 8 * prop.multiProcessorCount;
    c->mlpGridL23 = 4 * prop.multiProcessorCount;
    c->mlpGridTrain = prop.multiProcessorCount;
    CS_CUDA(cudaFuncSetAttribute(cs_mlp_l1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_SMEM_L1));
    CS_CUDA(cudaFuncSetAttribute(cs_mlp_l23_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_SMEM_L23));
    CS_CUDA(cudaFuncSetAttribute(cs_mlp_bwd23_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_SMEM_BWD23));
    CS_CUDA(cudaFuncSetAttribute(cs_mlp_bwd1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_SMEM_BWD1));
    MlpDev& M = c->mlp;
    const long long N = c->B.N;
    cs_status st;
#define MA(field, n) \
    if ((st = dalloc(c, &M.field, (size_t)(n))) != CS_OK) return st;
    MA(w, MLP_P);
    MA(wb, MLP_P);
    MA(m, MLP_P);
    MA(v, MLP_P);
    MA(gpart, (long long)c->mlpGridTrain * MLP_P);
    MA(loss_part, c->mlpGridTrain);
    MA(stats, MLP_NSTAT);
    MA(feat, N * 16);
    MA(h1, N * 64);
    MA(z1, N * 64);
    MA(z2, N * 64);
    MA(z3, N * 64);
    MA(y, N * 3);
    MA(du2, N * 128);
    MA(dfeat, std::max(1LL, (long long)slots * N * 16));
    MA(dtarget, std::max(1LL, (long long)slots * N * 3));
    MA(pred, N * 3);
    MA(dy, N * 3);
    MA(epart, 2LL * c->B.n_slices);
    MA(sheet_c, c->B.S);
    MA(sheet_scale, 2LL * c->B.S);
    MA(sheet_loss, c->B.S);
    MA(err, 1);
#undef MA
    if ((st = dalloc(c, &c->mlpScratch, 4096 + MLP_P)) != CS_OK) return st;
    M.slots = slots;
    M.grid = c->mlpGridTrain;
    CS_CUDA(cudaMemset(M.err, 0, sizeof(int)));
    // initial weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)), output layer x0.1, zero biases
    std::vector<float> w(MLP_P, 0.0f);
    uint64_t rs = seed;
    auto uni = [&](float a) { return a * (2.0f * (float)((splitmix(rs) >> 11) * (1.0 / 9007199254740992.0)) - 1.0f); };
    for (int i = 0; i < 64 * 32; i++) w[MLP_W1 + i] = uni(1.0f / std::sqrt(32.0f));
    for (int i = 0; i < 64 * 128; i++) w[MLP_W2 + i] = uni(1.0f / std::sqrt(128.0f));
    for (int i = 0; i < 64 * 64; i++) w[MLP_W3 + i] = uni(1.0f / std::sqrt(64.0f));
    for (int i = 0; i < 3 * 64; i++) w[MLP_W4 + i] = 0.1f * uni(1.0f / std::sqrt(64.0f));
    if ((st = mlpUploadWeights(c, w)) != CS_OK) return st;
    std::vector<float> stats(MLP_NSTAT, 0.0f);
    for (int i = 0; i < 16; i++) stats[16 + i] = 1.0f;
    for (int i = 0; i < 3; i++) stats[35 + i] = 1.0f;
    CS_CUDA(cudaMemcpy(M.stats, stats.data(), MLP_NSTAT * sizeof(float), cudaMemcpyHostToDevice));
    c->mlpInit = true;
    return CS_OK;
}

cs_status cs_mlp_record(cs_ctx* c, int slot, int what) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    if (slot < 0 || slot >= c->mlp.slots || (what != 0 && what != 1)) return fail(c, CS_ERR_INVALID_ARG, "bad slot");
    Batch& B = c->B;
    float* f = c->mlp.dfeat + (size_t)slot * B.N * 16;
    if (what == 0)
        cs_mlp_features_kernel<<<nblk(B.N, 256), 256, 0, c->stream>>>(B, c->mlp, f);
    else
        cs_mlp_target_kernel<<<nblk(3LL * B.N, 256), 256, 0, c->stream>>>(B, f, c->mlp.dtarget + (size_t)slot * B.N * 3);
    CS_CUDA(cudaGetLastError());
    return CS_OK;
}

// Sums of the 16 features, the 3 targets and their squares over the recorded slots
// (38 doubles: 16 + 3 sums, then 16 + 3 sums of squares) and the node count.
cs_status cs_mlp_moments(cs_ctx* c, int n_slots, double* sums, long long* count) {
    if (!c || !sums) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    if (n_slots <= 0 || n_slots > c->mlp.slots) return fail(c, CS_ERR_INVALID_ARG, "bad slot count");
    CS_CUDA(cudaSetDevice(c->device));
    const int blocks = 296;
    double* part = nullptr;
    CS_CUDA(cudaMalloc(&part, (size_t)blocks * 38 * sizeof(double)));
    const long long n = (long long)n_slots * c->B.N;
    cs_mlp_moments_kernel<<<blocks, 128, 0, c->stream>>>(c->mlp.dfeat, c->mlp.dtarget, n, part);
    std::vector<double> h((size_t)blocks * 38);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(part);
    if (e != cudaSuccess) return fail(c, CS_ERR_CUDA, "moments: %s", cudaGetErrorString(e));
    for (int k = 0; k < 38; k++) sums[k] = 0.0;
    for (int b = 0; b < blocks; b++)
        for (int k = 0; k < 38; k++) sums[k] += h[38 * b + k];
    if (count) *count = n;
    return CS_OK;
}

// The input and output normalisation from moment sums (one rank's, or summed over ranks).
cs_status cs_mlp_set_moments(cs_ctx* c, const double* sum, long long n) {
    if (!c || !sum || n <= 0) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    std::vector<float> stats(MLP_NSTAT);
    for (int k = 0; k < 16; k++) {
        double mu = sum[k] / n, var = sum[19 + k] / n - mu * mu;
        stats[k] = (float)mu;
        stats[16 + k] = (float)std::max(std::sqrt(std::max(var, 0.0)), 1e-6 * std::max(std::fabs(mu), 1e-30) + 1e-30);
    }
    for (int k = 0; k < 3; k++) {
        double mu = sum[16 + k] / n, var = sum[35 + k] / n - mu * mu;
        stats[32 + k] = (float)mu;
        stats[35 + k] = (float)std::max(std::sqrt(std::max(var, 0.0)), 1e-12);
    }
    CS_CUDA(cudaMemcpy(c->mlp.stats, stats.data(), MLP_NSTAT * sizeof(float), cudaMemcpyHostToDevice));
    return CS_OK;
}

cs_status cs_mlp_fit_normalization(cs_ctx* c, int n_slots) {
    double sums[38];
    long long n = 0;
    cs_status st = cs_mlp_moments(c, n_slots, sums, &n);
    if (st != CS_OK) return st;
    return cs_mlp_set_moments(c, sums, n);
}

// One minibatch's gradient into a device buffer (for an all-reduce across ranks).
cs_status cs_mlp_gradient_device(cs_ctx* c, int slot, int s0, int s1, float* grad, float* loss) {
    if (!c || !grad) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    if (slot < 0 || slot >= c->mlp.slots || s0 < 0 || s1 <= s0 || s1 > c->B.S)
        return fail(c, CS_ERR_INVALID_ARG, "bad slot or sheet range");
    CS_CUDA(cudaSetDevice(c->device));
    float* acc = c->mlpScratch;
    CS_CUDA(cudaMemsetAsync(acc, 0, sizeof(float), c->stream));
    mlpForwardBackward(c, slot, s0, s1);
    cs_mlp_adam_kernel<<<nblk(MLP_P, 256), 256, 0, c->stream>>>(c->mlp, c->mlpGridTrain, 0.f, 0.f, 0.f, 0.f, 1, grad);
    cs_mlp_loss_acc_kernel<<<1, 32, 0, c->stream>>>(c->mlp, c->mlpGridTrain, acc);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    if (loss) CS_CUDA(cudaMemcpy(loss, acc, sizeof(float), cudaMemcpyDeviceToHost));
    return mlpCheckErr(c);
}

// The Adam step cs_mlp_train takes after each minibatch, with a given (device) gradient.
cs_status cs_mlp_apply_gradient(cs_ctx* c, const float* grad, float lr) {
    if (!c || !grad || !(lr > 0)) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    CS_CUDA(cudaSetDevice(c->device));
    c->adamStep++;
    cs_mlp_adam_ext_kernel<<<nblk(MLP_P, 256), 256, 0, c->stream>>>(c->mlp, grad, lr, 0.9f, 0.999f, 1e-8f,
                                                                     (int)c->adamStep);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    return mlpCheckErr(c);
}

cs_status cs_mlp_gradient(cs_ctx* c, int slot, int s0, int s1, float* grad, float* loss) {
    if (!c || !grad) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    if (slot < 0 || slot >= c->mlp.slots || s0 < 0 || s1 <= s0 || s1 > c->B.S)
        return fail(c, CS_ERR_INVALID_ARG, "bad slot or sheet range");
    float* acc = c->mlpScratch;
    float* gout = c->mlpScratch + 4096;
    CS_CUDA(cudaMemsetAsync(acc, 0, sizeof(float), c->stream));
    mlpForwardBackward(c, slot, s0, s1);
    cs_mlp_adam_kernel<<<nblk(MLP_P, 256), 256, 0, c->stream>>>(c->mlp, c->mlpGridTrain, 0.f, 0.f, 0.f, 0.f, 1, gout);
    cs_mlp_loss_acc_kernel<<<1, 32, 0, c->stream>>>(c->mlp, c->mlpGridTrain, acc);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    CS_CUDA(cudaMemcpy(grad, gout, MLP_P * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) CS_CUDA(cudaMemcpy(loss, acc, sizeof(float), cudaMemcpyDeviceToHost));
    return mlpCheckErr(c);
}

cs_status cs_mlp_train(cs_ctx* c, int n_slots, int epochs, float lr, int sheets_per_batch, unsigned long long seed,
                       float* epoch_loss) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    if (n_slots <= 0 || n_slots > c->mlp.slots || epochs <= 0 || epochs > 4096 || !(lr > 0) || sheets_per_batch <= 0)
        return fail(c, CS_ERR_INVALID_ARG, "bad training arguments");
    CS_CUDA(cudaSetDevice(c->device));
    const int S = c->B.S;
    const int groups = (S + sheets_per_batch - 1) / sheets_per_batch;
    std::vector<std::pair<int, int>> order;
    for (int sl = 0; sl < n_slots; sl++)
        for (int g = 0; g < groups; g++) order.push_back({sl, g});
    uint64_t rs = seed;
    float* acc = c->mlpScratch;
    CS_CUDA(cudaMemsetAsync(acc, 0, epochs * sizeof(float), c->stream));
    for (int ep = 0; ep < epochs; ep++) {
        for (size_t i = order.size(); i > 1; i--) std::swap(order[i - 1], order[splitmix(rs) % i]);
        for (auto& o : order) {
            const int s0 = o.second * sheets_per_batch, s1 = std::min(S, s0 + sheets_per_batch);
            mlpForwardBackward(c, o.first, s0, s1);
            c->adamStep++;
            cs_mlp_adam_kernel<<<nblk(MLP_P, 256), 256, 0, c->stream>>>(c->mlp, c->mlpGridTrain, lr, 0.9f, 0.999f,
                                                                       1e-8f, (int)c->adamStep, nullptr);
            cs_mlp_loss_acc_kernel<<<1, 32, 0, c->stream>>>(c->mlp, c->mlpGridTrain, acc + ep);
        }
    }
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    if (epoch_loss) {
        std::vector<float> h(epochs);
        CS_CUDA(cudaMemcpy(h.data(), acc, epochs * sizeof(float), cudaMemcpyDeviceToHost));
        for (int ep = 0; ep < epochs; ep++) epoch_loss[ep] = h[ep] / (float)order.size();
    }
    return mlpCheckErr(c);
}

cs_status cs_mlp_energy_begin(cs_ctx* c, const cs_step_params* p) {
    if (!c || !p) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    c->energyBegun = false;
    cs_status st = mlpEnergyPrepare(c, p);
    if (st != CS_OK) return st;
    c->energyBegun = true;
    c->energyLoopCap = toDev(p).loop_cap;
    return CS_OK;
}

cs_status cs_mlp_energy_gradient_device(cs_ctx* c, int s0, int s1, float* grad, float* loss) {
    if (!c || !grad) return CS_ERR_INVALID_ARG;
    if (!c->energyBegun) return fail(c, CS_ERR_STATE, "cs_mlp_energy_begin first");
    if (s0 < 0 || s1 <= s0 || s1 > c->B.S) return fail(c, CS_ERR_INVALID_ARG, "bad sheet range");
    float* acc = c->mlpScratch;
    CS_CUDA(cudaMemsetAsync(acc, 0, sizeof(float), c->stream));
    mlpEnergyForwardBackward(c, s0, s1);
    cs_mlp_energy_loss_kernel<<<1, 32, 0, c->stream>>>(c->mlp, s0, s1, acc);
    cs_mlp_adam_kernel<<<nblk(MLP_P, 256), 256, 0, c->stream>>>(c->mlp, c->mlpGridTrain, 0.f, 0.f, 0.f, 0.f, 1, grad);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    if (loss) CS_CUDA(cudaMemcpy(loss, acc, sizeof(float), cudaMemcpyDeviceToHost));
    return mlpCheckErr(c);
}

cs_status cs_mlp_energy_end(cs_ctx* c, cs_step_stats* stats) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->energyBegun) return fail(c, CS_ERR_STATE, "cs_mlp_energy_begin first");
    c->energyBegun = false;
    // the end of the step: dv = the solution, v and x updated when asked (cs_advance_kernel)
    cs_advance_kernel<<<nblk(3LL * c->B.N, 256), 256, 0, c->stream>>>(c->B);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    c->lastStepValid = true;
    c->steps++;
    if (stats) return fillStepStats(c, stats, c->energyLoopCap, false);
    return CS_OK;
}

cs_status cs_mlp_train_step(cs_ctx* c, const cs_step_params* p, float lr, int sheets_per_batch,
                            unsigned long long seed, cs_step_stats* stats, float* loss) {
    if (!c || !p || !(lr > 0) || sheets_per_batch <= 0) return CS_ERR_INVALID_ARG;
    cs_status st = cs_mlp_energy_begin(c, p);
    if (st != CS_OK) return st;
    const int S = c->B.S;
    const int groups = (S + sheets_per_batch - 1) / sheets_per_batch;
    std::vector<int> order(groups);
    for (int g = 0; g < groups; g++) order[g] = g;
    uint64_t rs = seed;
    for (int i = groups; i > 1; i--) std::swap(order[i - 1], order[splitmix(rs) % i]);
    float* acc = c->mlpScratch;
    CS_CUDA(cudaMemsetAsync(acc, 0, sizeof(float), c->stream));
    for (int g : order) {
        const int s0 = g * sheets_per_batch, s1 = std::min(S, s0 + sheets_per_batch);
        mlpEnergyForwardBackward(c, s0, s1);
        cs_mlp_energy_loss_kernel<<<1, 32, 0, c->stream>>>(c->mlp, s0, s1, acc);
        c->adamStep++;
        cs_mlp_adam_kernel<<<nblk(MLP_P, 256), 256, 0, c->stream>>>(c->mlp, c->mlpGridTrain, lr, 0.9f, 0.999f, 1e-8f,
                                                                   (int)c->adamStep, nullptr);
    }
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    if ((st = mlpCheckErr(c)) != CS_OK) {
        c->energyBegun = false;
        return st;
    }
    if (loss) {
        float h = 0.f;
        CS_CUDA(cudaMemcpy(&h, acc, sizeof(float), cudaMemcpyDeviceToHost));
        *loss = h / (float)groups;
    }
    return cs_mlp_energy_end(c, stats);
}

cs_status cs_mlp_energy_gradient(cs_ctx* c, const cs_step_params* p, int s0, int s1, float* grad, float* loss) {
    if (!c || !p || !grad) return CS_ERR_INVALID_ARG;
    if (!c->loaded) return fail(c, CS_ERR_STATE, "no batch loaded");
    if (s0 < 0 || s1 <= s0 || s1 > c->B.S) return fail(c, CS_ERR_INVALID_ARG, "bad sheet range");
    cs_status st = mlpEnergyPrepare(c, p);
    if (st != CS_OK) return st;
    float* acc = c->mlpScratch;
    float* gout = c->mlpScratch + 4096;
    CS_CUDA(cudaMemsetAsync(acc, 0, sizeof(float), c->stream));
    mlpEnergyForwardBackward(c, s0, s1);
    cs_mlp_energy_loss_kernel<<<1, 32, 0, c->stream>>>(c->mlp, s0, s1, acc);
    cs_mlp_adam_kernel<<<nblk(MLP_P, 256), 256, 0, c->stream>>>(c->mlp, c->mlpGridTrain, 0.f, 0.f, 0.f, 0.f, 1, gout);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaStreamSynchronize(c->stream));
    c->lastStepValid = false;
    c->energyBegun = false;
    CS_CUDA(cudaMemcpy(grad, gout, MLP_P * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) CS_CUDA(cudaMemcpy(loss, acc, sizeof(float), cudaMemcpyDeviceToHost));
    return mlpCheckErr(c);
}

cs_status cs_mlp_predict(cs_ctx* c, float* pred) {
    if (!c || !pred) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    float* d = c->B.z;  // solver scratch, free between steps
    launchMlpInference(c, d);
    CS_CUDA(cudaGetLastError());
    CS_CUDA(cudaMemcpyAsync(pred, d, 3 * (size_t)c->B.N * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CS_CUDA(cudaStreamSynchronize(c->stream));
    return mlpCheckErr(c);
}

cs_status cs_mlp_get_record(cs_ctx* c, int slot, float* feat, float* target) {
    if (!c) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    if (slot < 0 || slot >= c->mlp.slots) return fail(c, CS_ERR_INVALID_ARG, "bad slot");
    const size_t N = c->B.N;
    if (feat) CS_CUDA(cudaMemcpy(feat, c->mlp.dfeat + slot * N * 16, N * 16 * sizeof(float), cudaMemcpyDeviceToHost));
    if (target) CS_CUDA(cudaMemcpy(target, c->mlp.dtarget + slot * N * 3, N * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    return CS_OK;
}

cs_status cs_mlp_get_weights(cs_ctx* c, float* out, int n) {
    if (!c || !out || n != CS_MLP_PARAMS) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    CS_CUDA(cudaMemcpy(out, c->mlp.w, MLP_P * sizeof(float), cudaMemcpyDeviceToHost));
    CS_CUDA(cudaMemcpy(out + MLP_P, c->mlp.stats, MLP_NSTAT * sizeof(float), cudaMemcpyDeviceToHost));
    return CS_OK;
}

cs_status cs_mlp_set_weights(cs_ctx* c, const float* in, int n) {
    if (!c || !in || n != CS_MLP_PARAMS) return CS_ERR_INVALID_ARG;
    if (!c->mlpInit) return fail(c, CS_ERR_STATE, "cs_mlp_init first");
    for (int i = 0; i < n; i++)
        if (!std::isfinite(in[i])) return fail(c, CS_ERR_INVALID_ARG, "non-finite weight");
    std::vector<float> w(in, in + MLP_P);
    cs_status st = mlpUploadWeights(c, w);
    if (st != CS_OK) return st;
    CS_CUDA(cudaMemcpy(c->mlp.stats, in + MLP_P, MLP_NSTAT * sizeof(float), cudaMemcpyHostToDevice));
    return CS_OK;
}

}  // extern "C"
