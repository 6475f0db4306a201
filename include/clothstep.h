/* clothstep: a B200 (sm_100a) implementation of ClothSimulator's implicit cloth step.
 *
 * The reference has no C ABI: its implicit step is the C++ overload pair
 * Cloth::physicsStep(dt, gravity, wind, transformations, handleStiffness, proximities,
 * repulsionThickness) -- CPU (Cloth.cu:676-693, src/Cloth.cuh:91) and GPU (Cloth.cu:695-813,
 * src/Cloth.cuh:92) -- chosen by the global `gpu` flag set from `--gpu` (main.cu:7-29) and
 * called once per cloth from Simulator::physicsStep (Simulator.cu:578-586).  This header is the
 * seam that replaces the GPU overload: a context holds a batch of cloths ("sheets") resident in
 * HBM and advances all of them by one implicit step per call.
 *
 * Conventions: every function returns a cs_status; host arrays are owned by the caller and
 * copied in or out; device memory is owned by the context; one context per host thread.
 * cs_step is asynchronous on the context's stream (cs_sync waits).  No function falls back to
 * a CPU implementation: without a usable CUDA device cs_create returns CS_ERR_NO_DEVICE.
 */
#ifndef CLOTHSTEP_H
#define CLOTHSTEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cs_status {
    CS_OK = 0,
    CS_ERR_INVALID_ARG = 1,   /* bad sizes, indices out of range, NULL where required */
    CS_ERR_CUDA = 2,          /* a CUDA runtime call failed; see cs_last_error */
    CS_ERR_NOT_CONVERGED = 3, /* some instance stopped at its iteration cap (stats tell which) */
    CS_ERR_NON_SPD = 4,       /* a diagonal block is singular or a CG breakdown occurred */
    CS_ERR_TIMEOUT = 5,       /* the solve loop hit its trip bound */
    CS_ERR_STATE = 6,         /* call out of order (e.g. cs_step before cs_load_batch) */
    CS_ERR_NO_DEVICE = 7,     /* no CUDA device, or not an sm_100 device */
    CS_ERR_NOT_TRAINED = 8    /* learned warm start requested without a trained network */
} cs_status;

typedef struct cs_ctx cs_ctx;

/* Material as read by Material::Material (Material.cu:3-41): the data file's density, six
 * stretching rows of four values and 3x5 bending samples, and the cloth's multipliers. */
typedef struct cs_material_desc {
    float density;
    float stretching[6][4];
    float bending[3][5];
    float thicken, density_mult, stretching_mult, bending_mult;
} cs_material_desc;

/* One cloth.  Arrays follow Mesh::load's CPU branch (Mesh.cu:306-404): node positions and
 * velocities, uv vertices, and triangles as (node, uv-vertex) index triples.  Handles follow
 * Cloth::addHandles (Cloth.cu:653-664): the node's position at load is the target unless
 * handle_pos is given.  Wind follows Wind.cu:3-7; the reference has one global wind
 * (Simulator.cu:28), here each sheet has its own. */
typedef struct cs_sheet_desc {
    int n_nodes, n_verts, n_faces, n_handles;
    const float* x;            /* 3*n_nodes */
    const float* v;            /* 3*n_nodes, or NULL for zero velocity */
    const float* uv;           /* 2*n_verts */
    const int32_t* face_nodes; /* 3*n_faces */
    const int32_t* face_verts; /* 3*n_faces */
    const int32_t* handle_nodes; /* n_handles */
    const float* handle_pos;   /* 3*n_handles, or NULL */
    int material;              /* index into the materials passed to cs_load_batch */
    float wind_density, wind_drag, wind_velocity[3];
} cs_sheet_desc;

/* CS_PREC_PLAIN_FP32: FP32 PCG with FP32 dot products from the guess, stopping when its own
 * recursive residual meets tol (as the reference's solve does, Cloth.cu:784-788); its true
 * residual is then checked in FP64 and reported, and the sheet counts as converged only if that
 * meets tol.  CS_PREC_MIXED: FP32 PCG with FP64 dot products inside FP64 iterative
 * refinement until the FP64 residual b - A dv meets tol: whenever the recursive residual fell
 * by inner_tol, the FP64 residual replaces it and CG goes on with the same search direction
 * (reliable updates). */
enum { CS_PREC_PLAIN_FP32 = 0, CS_PREC_MIXED = 1 };
enum { CS_WARM_ZERO = 0, CS_WARM_PREVIOUS = 1, CS_WARM_LEARNED = 2, CS_WARM_GIVEN = 3 };

/* Parameters of one step (Cloth::physicsStep's dt, gravity, handleStiffness) plus solver
 * controls.  The reference's GPU solve stops at an absolute ||r|| < 1e-6 or 400 iterations
 * (Cloth.cuh:43-44); here the target is an FP64-checked relative residual. */
typedef struct cs_step_params {
    float dt;
    float gravity[3];
    float handle_stiffness;   /* Magic::handleStiffness, default 1e3 (Magic.cu:6) */
    double tol;               /* relative residual ||b - A dv|| / ||b||, checked in FP64 */
    double inner_tol;         /* mixed precision: residual reduction between FP64 residual
                                 replacements (reliable updates; 0: 1e-2) */
    int max_iters;            /* CG iterations per sheet per step */
    int sweep_cap;            /* mixed precision: CG iterations per sweep (0: no cap) */
    int precision;            /* CS_PREC_* */
    int warm_start;           /* CS_WARM_* */
    int advance;              /* 1: v += dv and x += dt v (a full step); 0: solve only */
    int use_graph;            /* 1: run the captured CUDA graph; 0: host-driven launches */
    int solver;               /* CS_SOLVER_*: which PCG kernels solve the sheets */
    int precond_degree;       /* cluster-resident solver's preconditioner: 0 or 1 the 3x3
                                 block-Jacobi inverse; an odd degree 3..CS_PRECOND_MAX_DEGREE a
                                 Chebyshev polynomial of that degree in the block-Jacobi-scaled
                                 matrix of each CTA's strip of rows (no exchange between CTAs).
                                 The batched loop uses block-Jacobi (with the coarse
                                 correction when `coarse`). */
    int coarse;               /* 1 adds a coarse-space correction, 0 leaves it out.  Cluster-resident
                                 solver with the Chebyshev preconditioner: one constant per
                                 component on each of a few geometric segments of every CTA's
                                 strip.  Batched loop: one per aggregate of about 256 nodes (the
                                 rest (u, v) binned into at most 16 x 16 cells), added to
                                 block-Jacobi; sheets with proximities keep block-Jacobi alone.
                                 Either way the coarse matrix R A R^T is inverted per sheet and
                                 step. */
    /* Cloth::physicsStep's `transformations` (Cloth.cuh:91-92): the motions' transformations at
     * this step (Simulator::updateTransformations, Simulator.cu:565-569), CS_TRANSFORM_FLOATS
     * floats each -- scaling, translation (3), rotation quaternion (s, x, y, z) -- as
     * Transformation holds them (Transformation.cu:3-19, Quaternion.cu:7-15).  A handle with a
     * motion (cs_set_handle_motions) pulls its node toward transformations[motion] applied to
     * its position at load (Transformation::applyToPoint, Transformation.cu:82-84;
     * Cloth::addHandleForces, Cloth.cu:157-169).  NULL / 0 when no handle moves. */
    const float* transformations;
    int n_transformations;    /* at most CS_MAX_MOTIONS */
    int warm_scale;           /* 1: a warm start d is first replaced, per sheet, by its Galerkin
                                 multiple (d^T b / d^T A d) d -- the multiple of d nearest to
                                 the solution in the energy norm, never farther than the zero
                                 guess -- before the guard compares its FP64 residual with the
                                 zero guess's (a sheet with d^T A d <= 0 discards it); 0: the
                                 warm start as given.  No counterpart in the reference. */
} cs_step_params;

#define CS_TRANSFORM_FLOATS 8
#define CS_MAX_MOTIONS 64

#define CS_PRECOND_MAX_DEGREE 15

/* CS_SOLVER_AUTO: sheets whose system fits one thread-block cluster's shared memory are
 * solved by a cluster each, the system resident on chip for the whole solve; the others by
 * the batched loop.  CS_SOLVER_BATCHED: every sheet by the batched loop (the system streamed
 * from HBM every iteration).  Both run the same mixed/plain PCG to the same FP64-checked
 * tolerance. */
#define CS_SOLVER_AUTO 0
#define CS_SOLVER_BATCHED 1

typedef struct cs_step_stats {
    int n_instances;
    int converged;            /* instances that met tol */
    int max_iters;            /* max CG iterations over instances */
    long long total_iters;    /* sum of CG iterations over instances */
    int max_sweeps;           /* max FP64 residual evaluations */
    int warm_rejected;        /* instances whose warm start was discarded */
    int loop_trips;           /* trips of the batched solve loop */
    double max_rel_residual;  /* max over instances of the final FP64 relative residual */
    float ms;                 /* device time of the step (CUDA events) */
} cs_step_stats;

/* Context lifetime (replaces the per-cloth cuBLAS/cuSPARSE handles, Cloth.cu:19-20). */
cs_status cs_create(cs_ctx** ctx, int device);
cs_status cs_destroy(cs_ctx* ctx);
const char* cs_last_error(const cs_ctx* ctx);

/* Uploads a batch of cloths: topology (Mesh::load, Mesh.cu:306-452), face rest data
 * (Face::initialize, Face.cu:12-20), lumped masses (Mesh.cu:182-203), material tables
 * (Material.cu:3-41), handles, and the fixed block-sparse pattern of the system. */
cs_status cs_load_batch(cs_ctx* ctx, const cs_material_desc* materials, int n_materials,
                        const cs_sheet_desc* sheets, int n_sheets);

/* sizes[0..6] = nodes, faces, interior edges, stored 3x3 blocks (incl. padding), slices,
 * sheets, nonzero blocks of the system (the mesh pattern's, plus proximity blocks outside
 * it while proximities are set). */
cs_status cs_get_sizes(const cs_ctx* ctx, long long* sizes);

/* info[0..10] = sheets solved cluster-resident, CTAs per cluster, threads per CTA, clusters
 * in the persistent grid, SELL panels per CTA in shared memory, dynamic shared memory bytes
 * per CTA; the batched SpMV's launch shape (threads per block, slices per warp, slots loaded
 * together; cs_tune); the fastest resident preconditioner cs_tune found (degree, coarse
 * correction; 0, 0 before tuning).  No counterpart in the reference (its solver has no plan). */
cs_status cs_get_solver_info(const cs_ctx* ctx, int* info);

/* --- Autotuner ------------------------------------------------------------------------------
 * No counterpart in the reference, whose GPU solve calls cuSPARSE's COO SpMV with its default
 * algorithm (Cloth.cu:767-778, 790).  cs_tune times, with CUDA events on the context's stream and
 * on the loaded batch's system for the current state (params as for cs_step): every launch shape
 * of the batched SpMV -- threads per block, SELL slices per warp, block slots whose loads are
 * issued together -- reps launches each, and whole cluster-resident solves with each
 * preconditioner (block-Jacobi; strip-local Chebyshev of degree 3, 5 and 7 without and with the
 * coarse-space correction; one untimed, then the mean of min(reps, 3)), then whole solves by
 * either route (resident sheets on the cluster kernel and the rest in the batched loop, or all
 * in the batched loop; one untimed, then the mean of min(reps, 2)).  Every SpMV shape computes the same bits (out->spmv_checksum holds a
 * checksum of each shape's output); the fastest is used by the following steps.  The fastest
 * preconditioner is reported (cs_get_solver_info info[9], info[10]) for the caller's
 * cs_step_params.precond_degree / coarse, and the faster route (out->best_solver) for its
 * cs_step_params.solver.  Overwrites the solver's scratch vectors (not x, v, dv);
 * out may be NULL. */
#define CS_TUNE_SPMV_SHAPES 24
#define CS_TUNE_PRECONDS 6
typedef struct cs_tune_result {
    float spmv_ms[CS_TUNE_SPMV_SHAPES];
    uint32_t spmv_checksum[CS_TUNE_SPMV_SHAPES];
    int spmv_threads[CS_TUNE_SPMV_SHAPES], spmv_spw[CS_TUNE_SPMV_SHAPES], spmv_unroll[CS_TUNE_SPMV_SHAPES];
    float precond_ms[CS_TUNE_PRECONDS];  /* 0 when no sheet is solved cluster-resident */
    int precond_degree[CS_TUNE_PRECONDS], precond_coarse[CS_TUNE_PRECONDS];
    int best_spmv, best_precond;         /* indices; best_precond -1 without resident sheets */
    /* one whole solve of the system, with the fastest preconditioner: [0] CS_SOLVER_AUTO (0
     * without resident sheets), [1] CS_SOLVER_BATCHED; best_solver = the faster one's code */
    float solver_ms[2];
    int best_solver;
} cs_tune_result;
cs_status cs_tune(cs_ctx* ctx, const cs_step_params* params, int reps, cs_tune_result* out);

/* out[0..2] = 3x3 blocks of the systems of the sheets now solved cluster-resident (the mesh
 * pattern's), those among them whose row and column belong to the same CTA's strip of rows
 * (what one strip-local SpMV of the Chebyshev preconditioner reads), and the power iterations
 * each resident solve runs for that preconditioner's eigenvalue bound.  For work accounting
 * (rooflines); no counterpart in the reference. */
cs_status cs_get_resident_blocks(const cs_ctx* ctx, long long* out);

/* Node state of the whole batch, sheets concatenated in load order (3 floats per node). */
cs_status cs_set_state(cs_ctx* ctx, const float* x, const float* v);

/* The motion of every handle (Handle::motionIndex, Handle.cuh:9-16, from a scene's
 * "handles"[].motion, Simulator.cu:104-111): n = the handles of all sheets in load order, each
 * sheet's in its handle_nodes order; -1 = fixed at its target (the default after cs_load_batch).
 * Each step then takes the motions' transformations from cs_step_params.transformations. */
cs_status cs_set_handle_motions(cs_ctx* ctx, const int32_t* motion, int n);

/* One proximity as Cloth::physicsStep receives it (Proximity.cuh:11-21; built by the
 * collision detection the reference runs before the step, Simulator.cu:300-349): four
 * points with weights w (vertex-face: 1 and minus the face point's barycentric weights;
 * edge-edge: 1-s, s, -(1-t), -t), a unit normal, a friction coefficient and a stiffness
 * already scaled by the smaller area (Proximity.cu:5-24).  nodes[i] is a node of the batch
 * (its sheet's node_off + local index) or -1 for a point outside the batch (an obstacle's
 * node), whose position, velocity, mass and free flag (bit i of free_mask) are given here. */
typedef struct cs_proximity_desc {
    int nodes[4];
    float x[4][3];
    float v[4][3];
    float mass[4];
    int free_mask;
    float normal[3];
    float w[4];
    float mu;
    float stiffness;
} cs_proximity_desc;

/* Proximities of the following steps (until the next call; n = 0 clears them) and the
 * repulsion thickness (Magic::repulsionThickness, Magic.cu:9).  Each step then adds the
 * repulsion and friction terms of Cloth::addProximityForces (Cloth.cu:171-192) to every
 * sheet that holds one of a proximity's nodes, after the handle terms, in proximity order;
 * nodes of other sheets enter a sheet's terms through their state at the start of the step
 * (the reference steps cloths one after another, so a later cloth there sees an earlier
 * cloth's updated velocities).  Blocks outside the mesh's pattern are kept beside it;
 * cs_get_system returns them merged.  Sheets with proximities are solved by the batched
 * loop. */
cs_status cs_set_proximities(cs_ctx* ctx, const cs_proximity_desc* proximities, int n, float thickness);

/* Proximity detection: what Simulator::physicsStep runs before stepping the cloths
 * (Simulator.cu:571-586, findProximitiesGpu Simulator.cu:300-349).  Every pair of faces of
 * sheets in one collision group whose bounds overlap after dilating one of them by
 * 2 x repulsion_thickness is tested for vertex-face and edge-edge proximity
 * (Simulator.cu:198-269); per (node | edge | face, side) the nearest candidate is kept
 * (ties: the lower element index), and those nearer than 2 x repulsion_thickness become
 * proximities (Proximity.cu:5-21) in the reference's order -- node keys, edge keys, face keys,
 * by element index and side.  They replace the set in force as cs_set_proximities does, with
 * repulsion_thickness as its thickness.  Runs on the device; *count receives the number. */
typedef struct cs_detect_params {
    float repulsion_thickness; /* Magic::repulsionThickness, default 1e-3 (Magic.cu:8) */
    float collision_stiffness; /* Magic::collisionStiffness, default 1e9 (Magic.cu:7) */
    float friction;            /* the scene's "friction", default 0.6 (Simulator.cu:25) */
    const int* sheet_group;    /* per sheet; sheets with equal groups interact.  NULL: all
                                  sheets interact, as the cloths of one scene */
} cs_detect_params;
cs_status cs_detect_proximities(cs_ctx* ctx, const cs_detect_params* params, int* count);

/* The proximities in force (set or detected): up to cap records; *count receives how many
 * there are. */
cs_status cs_get_proximities(cs_ctx* ctx, cs_proximity_desc* out, int cap, int* count);

/* The collision step Simulator::simulateStep runs after every physics step
 * (Simulator::collisionStep, Simulator.cu:602-684): rounds of continuous impact detection
 * between each node's position at the start of the last cs_step (x0) and its current one
 * (CollisionHelper.cu:3-136), selection of independent impacts by impact time
 * (Simulator.cu:394-420), and projection of the positions onto the impacts' constraints
 * (optimization/CollisionOptimization.cu, Optimization.cu); then v = (x - x0) / dt for
 * every node (Mesh.cu:238-247).  On the device.  CS_ERR_NOT_CONVERGED when impacts remain
 * after 2 x 100 rounds (the reference exits). */
typedef struct cs_collision_params {
    float thickness;         /* Magic::collisionThickness, default 1e-4 (Magic.cu:9-16) */
    float dt;                /* the step's time step */
    const int* sheet_group;  /* as in cs_detect_params */
} cs_collision_params;
typedef struct cs_collision_stats {
    int rounds;   /* detection rounds run */
    int impacts;  /* independent impacts projected */
} cs_collision_stats;
cs_status cs_collision_step(cs_ctx* ctx, const cs_collision_params* params, cs_collision_stats* stats);
cs_status cs_get_state(cs_ctx* ctx, float* x, float* v);
/* Same with device pointers (no host copy). */
cs_status cs_set_state_device(cs_ctx* ctx, const float* x, const float* v);
cs_status cs_get_state_device(cs_ctx* ctx, float* x, float* v);

/* One implicit step of every sheet: assemble (M - dt^2 df/dx) dv = dt (f + dt df/dx v)
 * (Cloth.cu:676-684), solve with batched PCG, and (if params->advance) v += dv, x += dt v
 * (Cloth.cu:690-692, Mesh.cu:226-231).  stats may be NULL.  Returns CS_ERR_NOT_CONVERGED if any
 * sheet stopped at its cap (the step is still applied). */
cs_status cs_step(cs_ctx* ctx, const cs_step_params* params, cs_step_stats* stats);
cs_status cs_sync(cs_ctx* ctx);

/* Warm start for CS_WARM_GIVEN: 3 floats per node (host). */
cs_status cs_set_warm_start(cs_ctx* ctx, const float* dv);
/* The last step's dv (3 floats per node, host). */
cs_status cs_get_dv(cs_ctx* ctx, float* dv);
/* Per-instance results of the last step: iterations, FP64 relative residual, flags
 * (1 converged, 2 warm start rejected, 4 breakdown, 8 iteration cap), each n_sheets long. */
cs_status cs_get_instance_stats(cs_ctx* ctx, int* iters, double* rel_residual, int* flags);

/* --- Inspection entry points used by the parity tests ------------------------------------ */

/* Assembles the system for the current state without solving (params->dt, gravity,
 * handle_stiffness are used). */
cs_status cs_assemble(cs_ctx* ctx, const cs_step_params* params);
/* The assembled system in block-CSR, rows = nodes in load order, columns sorted:
 * row_ptr (N+1), col (nnzb), val (9*nnzb, row-major blocks), b (3N), each may be NULL.
 * nnzb = sizes[6] of cs_get_sizes. */
cs_status cs_get_system(cs_ctx* ctx, int32_t* row_ptr, int32_t* col, float* val, float* b);
/* Per-element forces and Jacobians of the last assembly, expanded from the element records:
 * faces (9 and 81 floats each, PhysicsHelper.cu:264-291) and interior edges in the
 * reference's edge order (12 and 144 floats each, PhysicsHelper.cu:327-353); any may be NULL.
 * edge_nodes receives 4 node ids per interior edge. */
cs_status cs_get_element_forces(cs_ctx* ctx, float* face_f, float* face_J, float* edge_f, float* edge_J,
                                int32_t* edge_nodes);
/* y = A x with the assembled system (host vectors of 3N floats). */
cs_status cs_spmv(cs_ctx* ctx, const float* x, float* y);
/* Device pointers of the batch state, for zero-copy callers: x, v, dv (3N floats each). */
cs_status cs_device_pointers(cs_ctx* ctx, float** x, float** v, float** dv);

/* --- Measurement entry points --------------------------------------------------------------
 * The reference's only instrumentation is per-phase wall clock after cudaDeviceSynchronize
 * (Simulator.cu:845-855); these time on the device instead. */

/* Times each kernel of the step in isolation with CUDA events on the context's stream, `reps`
 * launches each, on the current batch: ms[0] 0 (the face terms are evaluated inside the
 * assembly gather), [1] edge (bending geometry), [2] gather (assembly),
 * [3] SpMV of a CG iteration, [4] vector update of a CG iteration, [5] per-instance reduction,
 * [6] FP64 residual SpMV, [7] one cluster-resident solve of all resident sheets (0 if none;
 * when every sheet is resident, cs_get_instance_stats then reports that solve), [8] the set-up
 * of its coarse-space correction (forming and inverting the coarse matrices; 0 without it),
 * [9] the batched loop's coarse set-up for the sheets the loop solves (forming and inverting
 * their coarse matrices), [10] one loop trip's coarse-correction kernels (0 without the
 * correction); ms holds 11 floats.  Overwrites the solver's scratch vectors and dv64 (not x, v
 * or dv). */
cs_status cs_profile_kernels(cs_ctx* ctx, const cs_step_params* params, int reps, float* ms);
/* Cumulative counts since cs_load_batch: [0] steps, [1] solve-loop trips, [2] kernel launches. */
cs_status cs_get_counters(cs_ctx* ctx, long long* counters);
/* The cudaStream_t the context launches on (for callers that record events on it). */
cs_status cs_get_stream(cs_ctx* ctx, void** stream);
/* The order the collision step gives n impacts (node ids nodes[4 i .. 4 i + 3], time t[i] >= 0,
 * type[i] 0 vertex-face / 1 edge-edge): by time (-0.0 as +0.0), then node ids, then type (the
 * reference's std::sort in Simulator::independentImpacts, Simulator.cu:394-420, ordered by
 * time; the rest makes the order total), then input index, computed by the same device sort
 * (four stable radix passes).  order[k] = the index of the k-th impact.  For tests; the
 * context must hold a batch (its collision scratch is used). */
cs_status cs_impact_order(cs_ctx* ctx, const int32_t* nodes, const float* t, const int32_t* type, int n,
                          int32_t* order);

/* Check of the tcgen05 tile GEMM the learned warm start is built on (no reference counterpart):
 * D[128 x N] = A[128 x K] * B[N x K]^T with BF16 inputs (raw 16-bit patterns, row-major host
 * arrays) and FP32 accumulation in tensor memory; K and N multiples of 16 in [16, 128]. */
cs_status cs_tc_gemm_check(const uint16_t* A, const uint16_t* B, float* D, int K, int N);

/* --- Learned warm start ---------------------------------------------------------------------
 * No counterpart in the reference.  A one-ring message-passing MLP predicts each step's dv
 * from per-node features of the assembled system (b, the diagonal block, v, the previous dv,
 * the mass); the batched solver starts from the prediction (cs_step with CS_WARM_LEARNED) and
 * discards it, per sheet, when its FP64 residual exceeds the zero guess's.  The layers run on
 * tcgen05 tensor cores (BF16 operands, FP32 accumulation).  Training is on the device:
 *   for each step of a trajectory: cs_assemble; cs_mlp_record(slot, 0); cs_step;
 *   cs_mlp_record(slot, 1); then cs_mlp_fit_normalization and cs_mlp_train. */
#define CS_MLP_PARAMS 14761  /* weights and biases (14723) + input/output normalisation (38) */
cs_status cs_mlp_init(cs_ctx* ctx, int dataset_slots, unsigned long long seed);
/* what = 0: features of the system assembled by the last cs_assemble (with the previous dv);
 * what = 1: the target (the last cs_step's dv minus that previous dv). */
cs_status cs_mlp_record(cs_ctx* ctx, int slot, int what);
cs_status cs_mlp_fit_normalization(cs_ctx* ctx, int n_slots);
/* Adam over minibatches of sheets_per_batch whole sheets of each recorded slot, shuffled per
 * epoch; epoch_loss (optional, epochs floats) receives the mean minibatch loss. */
cs_status cs_mlp_train(cs_ctx* ctx, int n_slots, int epochs, float lr, int sheets_per_batch,
                       unsigned long long seed, float* epoch_loss);
/* Gradient (CS_MLP_PARAMS - 38 floats) and loss of one minibatch, without updating. */
cs_status cs_mlp_gradient(cs_ctx* ctx, int slot, int sheet_begin, int sheet_end, float* grad, float* loss);
/* Energy-norm training on the solver's own trajectory, one step at a time (the normalisation
 * set first, e.g. by cs_mlp_fit_normalization on a few recorded steps).  cs_mlp_train_step is
 * one implicit step of the batch as cs_step takes it with `params` (assembly, the solve from
 * its zero or previous-dv start -- not the learned one -- then v and x updated when
 * params->advance), and between the solve and the update, for every minibatch of
 * sheets_per_batch whole sheets (in an order shuffled by seed), one Adam step on the loss
 *     L = mean over the minibatch's sheets of 1 - (p^T b)^2 / ((p^T A p)(dv*^T b))
 * of the network's prediction p for this step's system, dv* the step's solution (A dv* = b to
 * the solve's tolerance): sin^2 of the angle between p and dv* in the energy inner product,
 * i.e. the squared energy-norm error of p's Galerkin multiple (the start warm_scale makes of p)
 * relative to the zero guess's; in [0, 1], and its gradient needs one SpMV of the prediction.
 * *loss (optional) receives the mean of the minibatches' losses before their updates; stats as
 * cs_step's.
 * Batches with proximities are refused.  cs_mlp_energy_gradient: the same loss's gradient
 * (CS_MLP_PARAMS - 38 floats) and value for sheets [sheet_begin, sheet_end) of the current
 * state, without updating the weights or the state. */
cs_status cs_mlp_train_step(cs_ctx* ctx, const cs_step_params* params, float lr, int sheets_per_batch,
                            unsigned long long seed, cs_step_stats* stats, float* loss);
cs_status cs_mlp_energy_gradient(cs_ctx* ctx, const cs_step_params* params, int sheet_begin, int sheet_end,
                                 float* grad, float* loss);
/* cs_mlp_train_step in parts, for data-parallel training across ranks (each on its own
 * trajectories): cs_mlp_energy_begin (assembly, features, solve), then per minibatch of the
 * common schedule cs_mlp_energy_gradient_device (the loss's gradient for sheets
 * [sheet_begin, sheet_end) into a DEVICE buffer of CS_MLP_PARAMS - 38 floats, to all-reduce,
 * and the minibatch's loss) and cs_mlp_apply_gradient, then cs_mlp_energy_end (the state
 * update; stats as cs_step's).  With one rank and cs_mlp_train_step's minibatch order (its
 * seeded shuffle of the minibatches) they give its weights bit for bit. */
cs_status cs_mlp_energy_begin(cs_ctx* ctx, const cs_step_params* params);
cs_status cs_mlp_energy_gradient_device(cs_ctx* ctx, int sheet_begin, int sheet_end, float* grad, float* loss);
cs_status cs_mlp_energy_end(cs_ctx* ctx, cs_step_stats* stats);
/* Data-parallel training across ranks (one context per GPU, each on its own trajectories):
 * cs_mlp_moments gives the normalisation's sums (38 doubles: 16 feature and 3 target sums, then
 * their 19 sums of squares) and node count for an all-reduce, cs_mlp_set_moments sets the
 * normalisation from the summed moments (cs_mlp_fit_normalization = the two on one rank);
 * cs_mlp_gradient_device writes one minibatch's gradient into a DEVICE buffer of
 * CS_MLP_PARAMS - 38 floats (to all-reduce in place, e.g. with NCCL) and cs_mlp_apply_gradient
 * takes the Adam step cs_mlp_train takes after each minibatch, with that buffer's gradient. */
cs_status cs_mlp_moments(cs_ctx* ctx, int n_slots, double* sums, long long* count);
cs_status cs_mlp_set_moments(cs_ctx* ctx, const double* sums, long long count);
cs_status cs_mlp_gradient_device(cs_ctx* ctx, int slot, int sheet_begin, int sheet_end, float* grad, float* loss);
cs_status cs_mlp_apply_gradient(cs_ctx* ctx, const float* grad, float lr);
/* The prediction for the system assembled by the last cs_assemble (3 floats per node). */
cs_status cs_mlp_predict(cs_ctx* ctx, float* pred);
/* A recorded training pair: 16 raw features and 3 target values per node (host arrays). */
cs_status cs_mlp_get_record(cs_ctx* ctx, int slot, float* feat, float* target);
cs_status cs_mlp_get_weights(cs_ctx* ctx, float* out, int n);
cs_status cs_mlp_set_weights(cs_ctx* ctx, const float* in, int n);

/* --- Allocation-free solve ------------------------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory (a host
 * whose own allocator owns all device memory, real-time loops that must not allocate, plugins
 * that may not grow the device footprint): solves one 3x3-block CSR system A x = b with the
 * batched solver's scheme (FP32 block-Jacobi PCG, FP64 dots, FP64 iterative refinement to the
 * relative residual tol), using a fixed 2 MiB static device array as scratch instead of
 * allocating.  row_ptr (n_rows+1), col (nnzb), val (9*nnzb, row-major blocks), b and x (3*n_rows)
 * are device pointers owned by the caller; stream is a cudaStream_t (NULL = default stream).
 * n_rows above CS_NOALLOC_MAX_ROWS is rejected with CS_ERR_INVALID_ARG, as are out-of-range
 * row pointers or columns.  Every call on a device shares the one scratch array: calls that
 * overlap on the GPU race and must be serialised.  The first call on each device looks up the
 * array's address (cudaGetSymbolAddress) with that device current; make it before any stream
 * capture.  Two forms:
 *   - synchronous (iters or rel_residual, host pointers, given): the call waits for the stream
 *     and returns CS_OK, CS_ERR_NOT_CONVERGED (the iteration cap was reached; x holds the last
 *     iterate) or CS_ERR_INVALID_ARG (the device found a row pointer or column out of range;
 *     x is then NaN);
 *   - asynchronous (both NULL): the call returns after the launch, with CS_OK or an error of
 *     the arguments or of the launch only.  The device's own checks and the convergence are
 *     not reported to this form: a rejected system leaves NaN in x, and a caller that needs
 *     the status uses the synchronous form. */
#define CS_NOALLOC_MAX_ROWS 16384
cs_status cs_solve_block_csr_noalloc(int n_rows, int nnzb, const int32_t* row_ptr, const int32_t* col,
                                     const float* val, const float* b, float* x, double tol, int max_iters,
                                     void* stream, int* iters, double* rel_residual);

#ifdef __cplusplus
}
#endif

#endif /* CLOTHSTEP_H */
