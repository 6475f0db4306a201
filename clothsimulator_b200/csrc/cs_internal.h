// Internal data layout of the B200 implicit cloth step.  Not part of the C ABI.
//
// HBM layout (one batch of independent sheets = "instances"):
//   nodes   : x, v, dv as 3N floats (xyz interleaved), mass N, handle float4 N (xyz target,
//             w = handle count), FP64 solution accumulator dv64 3N.
//   faces   : int4 {n0, n1, n2, sheet} (global node ids), float4 inverse rest matrix
//             (Face::inverse, Face.cu:16), rest area.
//   edges   : interior edges only (the reference skips boundary edges, Cloth.cu:142):
//             int4 {n0, n1, opposite0, opposite1}, int meta (face-vertex rotations), sheet,
//             float4 {area0 + area1, bias weight side 0, side 1, 0}; per step a 64-byte
//             record of its bending geometry (dtheta, coefficient, theta).
//   system  : SELL-32 block layout.  A sheet's rows (nodes), sorted by block count within
//             windows of sigma rows (sigma chosen per topology to minimise padding), are cut
//             into slices of 32; slice s has `width` block slots per row (padded with zero
//             blocks).  Slot (slice, k, lane) stores its 3x3 block in a "panel" of 32 lanes:
//             entries 0-3 as float4[32], entries 4-7 as float4[32], entry 8 as float[32]
//             (1152 bytes per panel, 128-bit coalesced loads).  Slot k = 0 is the diagonal.
//             Column indices and the assembly's row lists are per *topology* (shared by all
//             sheets with identical connectivity) and hold sheet-local ids.
#ifndef CLOTHSTEP_CS_INTERNAL_H
#define CLOTHSTEP_CS_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "clothstep.h"

#define CS_SLICE 32
#define CS_PANEL_FLOATS 288  // 32 lanes x 9 entries
#define CS_TABLE_N 30
#define CS_TABLE_ENTRIES (CS_TABLE_N * CS_TABLE_N * CS_TABLE_N)
// Contributor code: bit 31 = edge (1) / face (0); bits 4..30 = sheet-local element id;
// bits 2..3 = local row corner a; bits 0..1 = local column corner b.
#define CS_CODE_EDGE 0x80000000u
__host__ __device__ inline uint32_t cs_code(int is_edge, int elem, int a, int b) {
    return (is_edge ? CS_CODE_EDGE : 0u) | ((uint32_t)elem << 4) | ((uint32_t)a << 2) | (uint32_t)b;
}
// Threads per CTA of the assembly gather (forces.cu) at most; its slot accumulators take
// gather_width x 1152 bytes of shared memory per warp, and a batch whose widest slice would not
// fit four warps in a CTA's shared memory gets fewer.  (One-warp CTAs, 15 warps per SM instead
// of 12, measured slower on the windy batch: 3.82 against 3.35 ms.)
#define CS_GATHER_THREADS 128

struct SheetDesc {
    int node_off, n_nodes;
    int face_off, n_faces;
    int edge_off, n_edges;      // interior edges
    int slice_off, n_slices;    // global slices
    int topo;                   // shared topology id
    int table;                  // stretching table id
    float bending[15];          // scaled bending samples, 3x5 (Material.cu:38-40)
    float wind_density, wind_drag, wind_v[3];
    int nbr_ptr_off, nbr_off;   // this sheet's topology in the one-ring neighbour arrays
    int row2slot_off;           // this sheet's topology in the row -> slot map
    int resident;               // 1: solved by the cluster-resident kernel (resident.cu)
    int csr_ptr_off;            // this sheet's topology in tcsr_ptr (block CSR for slot lookups)
    int panel_off;              // first value panel: global slot = panel_off * 32 + topology slot
    // coarse space of the batched loop: this sheet's topology in the aggregate arrays, its
    // aggregates, its coarse unknowns' offset in the per-sheet vectors and its matrices' offset
    int bc_node_off, bc_agg_off, bc_mem_off, bc_pair_off, bc_npair, bc_na, bc_vec_off;
    long long bc_mat_off;
};

struct SliceDesc {
    int sheet;
    int topo_slice;  // index into the per-topology slice arrays
    int row0;        // the sheet's first node; lane l holds row row0 + rowmap[topo_slice * 32 + l]
    int rows;        // rows in this slice (<= 32)
    int width;       // block slots per row
    int panel0;      // first global value panel
    int tpanel0;     // first per-topology panel (columns, contributor lists)
    int pad;
};

// Solver phases of one instance (one sheet's system) inside the batched loop.
enum InstPhase : int {
    PH_CG = 0,        // one preconditioned CG iteration on the FP32 correction system
    PH_RES = 1,       // FP64 residual b - A (dv64 + e) and its norm
    PH_INIT = 2,      // start a CG sweep: dv64 += e, e = 0, z = P r, p = z (or, continuing after a
                      // reliable update, p = z + beta p with the FP64 residual in r)
    PH_FINISH = 3,    // dv64 += e, then done
    PH_DONE = 4,
    PH_RESIDENT = 5,  // owned by the cluster-resident kernel this step (skipped by the loop)
    PH_SCALE = 6,     // dv64 *= wscale (the warm start's Galerkin multiple), then PH_RES
};

// Cluster-resident solver limits: CTAs per cluster, warps (slices) per CTA, block slots per
// row (the SpMV over a row is fully unrolled to this width; column codes live in registers).
#define CS_RES_MAX_CL 16
#define CS_RES_MAX_WARPS 16
#define CS_RES_MAX_WIDTH 16
// Reliable updates keep the search direction only while the recursive residual has drifted
// from the FP64 one by at most this fraction of the latter (larger drift: restart).
#define CS_RELIABLE_DRIFT 0.1
#define CS_CHEB_POWER_ITERS 10
// A sheet uses the strip-local Chebyshev preconditioner only if at least this share of its
// blocks couple rows of one strip.  Small sheets split into thin strips do better with
// block-Jacobi; measured on the B200 (hanging and windy sheets, tol 1e-6): 24x24 (0.54 of the
// blocks strip-local) and 28x28 (0.59) need fewer or as many iterations with block-Jacobi, 32x32
// (0.71), 40x40 (0.65), 48x48 (0.84) and 64x64 (0.89) fewer with the Chebyshev polynomial.
#define CS_CHEB_MIN_LOCAL 0.62  // power iterations per sheet solve for the strip-local Chebyshev bound
// Coarse-space correction of the cluster-resident solver (with the strip-local Chebyshev
// preconditioner): each CTA's strip of rows is cut into K segments along the principal axis of
// its nodes' rest (uv) coordinates, K = min(CS_COARSE_MAX_K, CS_COARSE_AGGS / CTAs per cluster);
// the coarse space holds one constant per (segment, component).
// threads of the per-instance reduction kernels of the batched loop
#define CS_REDUCE_THREADS 256
// coarse-space correction of the batched loop (coarse.cu): a sheet's nodes binned by their rest
// (u, v) into g x g cells (g = round(sqrt(nodes / CS_BC_NODES_PER_AGG)), 1..CS_BC_MAX_G), the
// non-empty cells its aggregates; coarse systems up to CS_BC_SMALL_NC unknowns are inverted by
// one CTA in shared memory, larger ones by a cluster of CS_BC_CLUSTER CTAs
#define CS_BC_NODES_PER_AGG 256
#define CS_BC_MAX_G 16
#define CS_BC_MAX_NC (3 * CS_BC_MAX_G * CS_BC_MAX_G)
#define CS_BC_SMALL_NC 192
#define CS_BC_CLUSTER 16
#define CS_BC_THREADS 512
// Gauss-Jordan pivot blocks of the coarse inversion: CS_BC_PB aggregates, CS_BC_KB rows
#define CS_BC_PB 4
#define CS_BC_KB (3 * CS_BC_PB)
#define CS_COARSE_MAX_K 8
#define CS_COARSE_AGGS 54
// Threads of the per-sheet set-up kernel that forms and inverts the coarse matrix, and its
// dynamic shared memory: the nc x nc matrix with rows padded to 16 bytes, then one pivot block.
#define CS_COARSE_THREADS 512
__host__ __device__ inline int cs_coarse_ld(int nc) { return (nc + 3) & ~3; }
__host__ __device__ inline size_t cs_coarse_setup_smem(int nc) {
    return ((size_t)nc * cs_coarse_ld(nc) + CS_BC_KB * CS_BC_KB) * sizeof(float);
}
// Launch shapes of the batched SpMV that cs_tune times (pcg.cu, kSpmvShapes): threads per block,
// slices per warp, block slots whose loads are issued together.
struct SpmvShape {
    int threads, spw, unroll;
};
#define CS_SPMV_CANDIDATES 24
#define CS_SPMV_DEFAULT 1  // 128 threads, one slice per warp, no unrolling
struct Batch;
extern const SpmvShape kSpmvShapes[CS_SPMV_CANDIDATES];
void launchSpmvShape(const Batch& B, int shape, cudaStream_t st);
#define CS_SOLVER_AUTO_DEV 0
#define CS_SOLVER_BATCHED_DEV 1

// Instance flags
#define CS_IF_CONVERGED 1
#define CS_IF_WARM_REJECTED 2
#define CS_IF_BREAKDOWN 4
#define CS_IF_CAPPED 8

struct InstState {
    double bnorm2;      // ||b||^2 (FP64)
    double rz;          // r.z of the current iteration
    double rz_prev;     // r.z of the iteration before (a reliable update's beta)
    double pq;
    double rr;          // ||r||^2 of the recursive residual
    double res0;        // FP64 true residual norm at the start of the current sweep
    double resnorm;     // last FP64 true residual norm
    double first_res;   // FP64 residual of the initial guess
    float alpha, beta;
    int phase;
    int sweep_iters;
    int iters;          // total CG iterations this step
    int sweeps;         // FP64 residual evaluations this step
    int flags;
    int cont;           // the next PH_INIT keeps the search direction (reliable update)
    double wscale;      // Galerkin multiple of the warm start (warm_scale)
    int scaled;         // the warm start's scaling pass is done
    int pad;
};

// Step parameters in device memory (read by every kernel of the captured step graph).
struct DevParams {
    float dt;
    float gravity[3];
    float handle_stiffness;
    double tol;            // FP64-checked relative residual target
    double inner_tol;      // mixed precision: residual reduction between FP64 residual replacements
    int max_iters;         // CG iterations per instance per step
    int sweep_cap;         // CG iterations per sweep
    int mixed;             // 1: FP32 CG + FP64 refinement; 0: plain FP32 CG (FP32 dots)
    int warm;              // 0 zero guess, 1 warm start from dv64 as preloaded
    int loop_cap;          // hard bound on loop trips per step
    int advance;           // 1: v += dv, x += dt v at the end of the step
    int warm_scale;        // 1: the warm start replaced by its Galerkin multiple before the guard
    int solver;            // CS_SOLVER_AUTO_DEV: resident sheets on the cluster kernel; BATCHED: loop only
    int cheb_degree;       // resident solver: 1 block-Jacobi; odd >= 3 strip-local Chebyshev of that degree
    int coarse;            // resident solver with the Chebyshev preconditioner: 1 adds the coarse-space correction
    int n_motions;         // transformations of this step (cs_step_params.transformations)
    float motion[CS_MAX_MOTIONS][CS_TRANSFORM_FLOATS];
};

// One proximity as seen by one sheet it touches (cs_set_proximities): node[i] is a batch
// node or -1; bit i of `local` marks the nodes of this sheet (their rows and columns get
// blocks); other points enter through their state only.
struct ProxInst {
    int node[4];
    int local, free_mask, sheet;
    float thickness;
    float n[3], w[4], mu, stiffness;
    float xe[4][3], ve[4][3], me[4];  // points outside the batch (node -1)
};

// Per-instance record written by cs_prox_kernel: -dt^2 J of the impulse (12x12), -dt J of
// the friction (12x12), the impulse right-hand side dt (f + dt J v) (12), the friction one dt f.
#define CS_PROX_REC 312

struct Batch {
    int N = 0, F = 0, E = 0, S = 0;
    // coarse-space correction of the batched loop (coarse.cu)
    int bc_total_agg = 0;        // aggregates of all sheets (the per-aggregate kernels' work list)
    int bc_max_npair = 0;        // largest coarse pair count of a sheet
    int bc_n_big = 0;            // sheets whose coarse system exceeds CS_BC_SMALL_NC
    int2* bc_agg = nullptr;      // per global aggregate: (sheet, local aggregate)
    int* bc_big = nullptr;       // the sheets inverted by a cluster
    int* bc_node_agg = nullptr;  // per topology node: its aggregate
    int* bc_mptr = nullptr;      // per topology aggregate: member range (na + 1 per topology)
    int* bc_mem = nullptr;       // per topology: member nodes, by aggregate, ascending
    int4* bc_pair = nullptr;     // per topology coarse pair: (a, b, contributor begin, end)
    int* bc_contrib = nullptr;   // topology slots (panel * 32 + lane) of the stored blocks of each pair
    float* bc_mat = nullptr;     // per sheet nc x nc: the coarse matrix R A R^T (then GJ's work)
    float* bc_inv = nullptr;     // per sheet nc x nc: its inverse, symmetrised
    float* bc_rc = nullptr;      // per sheet nc: R r
    float* bc_ec = nullptr;      // per sheet nc: A_c^-1 R r
    int* bc_ok = nullptr;        // per sheet: the coarse inverse of this step is valid
    int n_slices = 0, n_panels = 0, n_tpanels = 0, n_tables = 0;
    // nodes
    float *x = nullptr, *v = nullptr, *dv = nullptr, *mass = nullptr;
    float* x0 = nullptr;     // positions at the start of the last step (Node::x0, Mesh.cu:226-231)
    float4* handle = nullptr;
    int* handle_motion = nullptr;  // per node: the motion of its handle (-1: fixed)
    double* dv64 = nullptr;
    float* warm = nullptr;   // warm-start vector (previous dv or learned prediction)
    // faces
    int4* face_nodes = nullptr;
    float4* face_inv = nullptr;
    float* face_area = nullptr;
    // edges
    int4* edge_nodes = nullptr;
    int* edge_meta = nullptr;
    int* edge_sheet = nullptr;
    float4* edge_par = nullptr;
    float4* edge_geo = nullptr;  // per step: 4 per edge, dtheta (12), coefficient, theta (cs_edge_kernel)
    // sheets, materials, topology
    SheetDesc* sheets = nullptr;
    float4* tables = nullptr;
    SliceDesc* slices = nullptr;
    int* tcol = nullptr;         // per topology panel: 32 local column ids
    // assembly row lists (forces.cu, cs_gather_kernel): per topology node (at row2slot_off),
    // its (face << 2 | corner, slots of the face's corners) in face order and its (interior
    // edge << 2 | corner, slots of the edge's four nodes) in edge order; slots 8 bits each
    int* rface_ptr = nullptr;    // topology nodes of all topologies + 1
    int2* rface = nullptr;
    int* redge_ptr = nullptr;
    int2* redge = nullptr;
    int gather_width = 0;        // widest slice of the batch (the gather's accumulators per lane)
    int* nbr_ptr = nullptr;      // per topology: one-ring neighbour CSR (sheet-local ids)
    int* nbr = nullptr;
    int* node_sheet = nullptr;   // sheet of every node
    int* rowmap = nullptr;       // per topology slice lane: sheet-local row
    int* row2slot = nullptr;     // per topology row: slice * 32 + lane
    // system
    float* A = nullptr;          // n_panels * 288
    float* b = nullptr;          // 3N
    float* Pinv = nullptr;       // 9N
    // PCG
    float *e = nullptr, *r = nullptr, *z = nullptr, *pA = nullptr, *pB = nullptr, *q = nullptr;
    double* part = nullptr;      // 2 per slice
    InstState* inst = nullptr;
    DevParams* params = nullptr;
    int* loop = nullptr;         // [0] loop trip counter, [1] instances not done, [5] resident work counter
    // cluster-resident solver (resident.cu)
    int n_resident = 0;          // sheets listed in rlist
    int res_cap = 0;             // panels per CTA held in shared memory
    int* rlist = nullptr;        // resident sheets, largest first
    int* rsplit = nullptr;       // per topology: CS_RES_MAX_CL + 1 sheet-relative slice bounds per CTA rank
    int* rcode = nullptr;        // per topology panel slot: index of its column in the reading CTA's p array
    int* rsendptr = nullptr;     // per topology: CS_RES_MAX_CL + 1 offsets into rsend per owner rank
    uint32_t* rsend = nullptr;   // halo sends: src slot | dst rank << 12 | dst halo index << 16
    int* rhalo = nullptr;        // per topology: CS_RES_MAX_CL + 1 halo slot counts per rank
    int* rcheb = nullptr;        // per topology and rank: 1 if the strip uses the Chebyshev preconditioner when asked
    int res_halo0 = 0;           // first halo slot of every CTA's p array (= own slots per CTA)
    int res_alt = 0;             // first slot of the second own-row buffer (strip-local Chebyshev)
    // coarse-space correction (resident.cu): per topology {coarse unknowns nc (0: none), segments
    // per strip K, first and last entry of the coarse pattern in cpair}; per topology row its
    // sheet-local aggregate (rank * K + segment; at row2slot offsets); per topology, rank and
    // warp the segments among the warp's rows (bit k: segment k); the coarse pattern's block
    // pairs {aggregate a, aggregate b, first, last contributor in ccontrib} with their stored
    // blocks as topology slots; per resident work item the inverse coarse matrix (nc x nc) and
    // whether it was formed.
    int4* rcoarse = nullptr;
    int* ragg = nullptr;
    int* rwmask = nullptr;       // per topology: CS_RES_MAX_CL x CS_RES_MAX_WARPS
    int4* cpair = nullptr;
    int* ccontrib = nullptr;
    float* cinv = nullptr;
    int* cvalid = nullptr;
    int res_cnc = 0;             // largest nc over the resident topologies (0: no coarse correction)
    int res_ck = 0;              // largest K
    int res_coff = 0;            // byte offset of the coarse region in the resident kernel's shared memory
    // per-topology block CSR (local ids, columns ascending) with the SELL slot of each block
    int* tcsr_ptr = nullptr;
    int* tcsr_col = nullptr;
    int* tcsr_slot = nullptr;
    // proximities (cs_set_proximities, cs_detect_proximities)
    int n_pinst = 0, n_px = 0;
    const ProxInst* pinst = nullptr;
    float* prec = nullptr;        // CS_PROX_REC per instance
    const int* prow_ptr = nullptr;   // N + 1: the instances holding each row's node
    const int* prow_inst = nullptr;  // ascending per row
    int* xptr = nullptr;          // N + 1: blocks outside the pattern, per row (null: none)
    int* xcol = nullptr;          // their columns (batch nodes), ascending per row
    float* xval = nullptr;        // 9 per block, summed each step
    int* sheet_prox = nullptr;    // per sheet: 1 if a proximity touches it (batched loop)
};

// Proximity detection (contact.cu, cs_detect_proximities).  Scene-wide ids: nodes and faces as
// in Batch, edges (every edge, not only interior ones) of all sheets concatenated in sheet order.
struct Contact {
    int E = 0;               // edges
    int n_keys = 0;          // 2 N + 2 E + 2 F
    int hash_bits = 0;       // grid buckets = 1 << hash_bits
    float repulsion = 0.f, stiffness = 0.f, friction = 0.f;
    float dilate = 0.f;      // bounds dilation of the candidate pairs (2 x repulsion; collision thickness)
    int ccd = 0;             // 1: face bounds over x0 and x (continuous impacts)
    const int4* face_edges = nullptr;  // 3 edges + collision group per face
    const int4* edges = nullptr;       // node 0, node 1, face side 0, face side 1
    const int* nf_ptr = nullptr;       // N + 1
    const int* nf_code = nullptr;      // face << 2 | corner, faces in index order
    const float* node_area = nullptr;  // Mesh::updateNodeGeometries (Mesh.cu:190-198)
    const float* edge_area = nullptr;  // Edge::area (Edge.cu:89-95)
    float* fn = nullptr;               // face normals (3 per face)
    float* nn = nullptr;               // node normals (3 per node)
    float* box = nullptr;              // face bounds: lo xyz, hi xyz
    unsigned* ext = nullptr;           // [0] largest face extent (float bits), [1] error flags
    int* head = nullptr;               // grid bucket heads (-1: empty)
    int* next = nullptr;               // 8 entries per face: next entry in the bucket
    unsigned long long* keys = nullptr;  // per (node|edge|face, side): distance bits << 32 | other id
    int2* pairs = nullptr;             // candidate face pairs (f, g > f)
    int pair_cap = 0;
    int* pair_count = nullptr;
    int* block_count = nullptr;        // compaction: valid keys per block, then exclusive offsets
    int* total = nullptr;
    cs_proximity_desc* out = nullptr;  // detected proximities
    int out_cap = 0;
};

// Collision step (collide.cu, cs_collision_step): continuous impacts and their projection.
struct ImpactRec {
    int nodes[4];
    float t, w[4], n[3];
    int type;  // 0 vertex-face, 1 edge-edge
    int pad[3];
};

struct Collide {
    float thickness = 0.f;
    ImpactRec* found = nullptr;   // impacts of this round
    int found_cap = 0;
    int* counters = nullptr;      // [0] impacts found, [1] impacts selected
    ImpactRec* sorted = nullptr;  // by time (then node ids)
    // radix sort of the found impacts: key and permutation double buffers, CUB temp storage
    unsigned long long *skey[2] = {nullptr, nullptr};
    int* sperm[2] = {nullptr, nullptr};
    void* stmp = nullptr;
    size_t stmp_bytes = 0;
    ImpactRec* all = nullptr;     // independent impacts accumulated this deformation level
    int* used = nullptr;          // per node: taken by a selected impact of this round
    int* nodemin = nullptr;       // per node: lowest live impact index touching it (selection)
    int* alive = nullptr;         // per found impact: still a candidate of the selection
    int* chosen = nullptr;        // per found impact (+1): selected, then its output offset
    // the projection's nodes and constraints
    int* mark = nullptr;          // N + 1: node in an impact, then its slot (exclusive scan)
    int* nodes = nullptr;         // slot -> node, ascending
    int* idx = nullptr;           // 4 per impact: slots of its nodes
    int* nptr = nullptr;          // slots + 1: each slot's constraint corners
    int* nfill = nullptr;
    int* nlist = nullptr;         // 4 impact + corner, ascending per slot
    float* x1 = nullptr;          // 3N: positions when the collision step began
    float *cur = nullptr, *next = nullptr, *grad = nullptr;  // 3 per slot
    float *lambda = nullptr, *coef = nullptr, *cterm = nullptr;  // per constraint
    float *nterm = nullptr, *gterm = nullptr;                  // per slot
};

#define CS_CONTACT_ITEMS 4096  // keys per compaction block (256 threads x 16)
#define CS_PAIR_STAGE 16       // candidate pairs staged per thread before appending
#define CS_SCAN_ITEMS 4096     // ints per block of the exclusive scan (1024 threads x 4)

#endif
