/*
 * admm_b200.h -- C ABI of the B200 ADMM substep backend (libadmm_b200.so).
 *
 * The library is a drop-in for the reference's GPU ADMM backend
 * (ADMMBackendGPU / ADMMImplGPU, src/solver/backend_gpu/admm_backend_gpu.h:13,
 * src/solver/backend_gpu/admm_impl_gpu.h:38) and its GPU collision detector
 * (BVH_GPU, src/contact/collision_detection_cuda.h:45).  Every entry point takes
 * plain pointers and sizes; host float buffers are row-major N x 3, the same
 * bytes as ADU::Matf_X3::data() (src/mutils/common_types.h:20,33).
 *
 * Every call returns 0 on success or a negative ADMM_ERR_* code; nothing in the
 * library exits the process (the reference exits on CUDA errors,
 * src/mutils/cuda_tools.cuh:37-46).  One handle owns one CUDA stream and all of
 * its device memory; calls on one handle must be serialised by the caller,
 * different handles are independent.
 */
#ifndef ADMM_B200_H
#define ADMM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ADMM_B200_ABI_VERSION 5

/* status codes */
#define ADMM_OK                    0
#define ADMM_ERR_INVALID          -1  /* bad argument / inconsistent description      */
#define ADMM_ERR_CUDA             -2  /* a CUDA runtime call failed                    */
#define ADMM_ERR_OOM              -3  /* device allocation failed                      */
#define ADMM_ERR_CONTACT_OVERFLOW -4  /* more contacts than max_contacts (clamped)     */
#define ADMM_ERR_STACK_OVERFLOW   -5  /* BVH traversal stack depth exceeded            */
#define ADMM_ERR_NAN              -6  /* non-finite value in the state                 */
#define ADMM_ERR_NOT_CONVERGED    -7  /* residual tolerance not reached at max_iter    */
#define ADMM_ERR_NO_DEVICE        -8  /* no usable sm_100 device                       */
#define ADMM_ERR_STATE            -9  /* call out of order (e.g. step before create)   */
#define ADMM_ERR_TIMEOUT         -10  /* a bounded device-side wait gave up            */

typedef struct AdmmB200 AdmmB200; /* opaque handle */

/*
 * Scene / constraint description.  Mirrors what ADMMImplGPU receives through
 * Solver::init(verts, mass, dt) (src/solver/solver.h:66-90),
 * add_constraints/addPins (solver.h:96,150), ADMMSolverConfig
 * (src/solver/core/admm_config.h:13-54) and the BVH_GPU geometry
 * (collision_detection_cuda.cpp:39-83).  Constraint rows are laid out as in
 * mesh_to_constraint.h:94-151: each type occupies a contiguous block of rows
 * starting at *_start_row (tri 2 rows, tet 3, bending 1, pin 1 per constraint).
 * All pointers are host pointers; the library copies what it needs in create.
 */
typedef struct AdmmB200Desc {
    int32_t abi_version;          /* ADMM_B200_ABI_VERSION */
    int32_t n_vert;               /* all vertices, dynamic first               */
    int32_t n_dyn;                /* static_vert_begin                         */
    int32_t n_rows;               /* m_nCDim (set_constraint_dim)               */
    const float*   x0;            /* [n_vert*3] initial positions               */
    const float*   v0;            /* [n_vert*3] initial velocities, may be NULL */
    const float*   mass;          /* [n_vert] lumped mass                       */
    const int32_t* is_fixed;      /* [n_vert] 1 = pinned (addPins), may be NULL */
    /* triangle strain (triangle_constraint.h:24-62) */
    int32_t n_tri, tri_start_row;
    const int32_t* tri_inds;      /* [n_tri*3] */
    const float*   tri_binv;      /* [n_tri*4] row-major 2x2 Binv */
    const float*   tri_w;         /* [n_tri]   w = sqrt(k*area)   */
    /* tetrahedral strain (tetrahedral_constraint.h:22-56) */
    int32_t n_tet, tet_start_row;
    const int32_t* tet_inds;      /* [n_tet*4] */
    const float*   tet_binv;      /* [n_tet*9] row-major 3x3 Binv */
    const float*   tet_w;         /* [n_tet]   w = sqrt(k*volume) */
    /* Laplacian bending (bending_constraint.h:24-78): CSR, entry 0 = middle vertex */
    int32_t n_bend, bend_start_row;
    const int32_t* bend_offsets;  /* [n_bend+1] */
    const int32_t* bend_inds;     /* [bend_offsets[n_bend]] */
    const float*   bend_coeffs;   /* [bend_offsets[n_bend]] D-row coefficients */
    const float*   bend_rest_norm;/* [n_bend] rest mean-curvature norm, may be NULL (= 0) */
    const float*   bend_w;        /* [n_bend] */
    /* pins (pin_constraint.h:18-57) */
    int32_t n_pin, pin_start_row;
    const int32_t* pin_inds;      /* [n_pin] */
    const float*   pin_pos;       /* [n_pin*3] */
    const float*   pin_w;         /* [n_pin] w = sqrt(k) */
    /* collision geometry (MeshData::surface_tris/_edges/_vinds) */
    int32_t n_surf_tri, n_surf_edge, n_surf_vert;
    const int32_t* surf_tris;     /* [n_surf_tri*3]  */
    const int32_t* surf_edges;    /* [n_surf_edge*2] */
    const int32_t* surf_verts;    /* [n_surf_vert]   */
    const float*   contact_w;     /* [n_vert] w_c per vertex (solver_config_applier.cpp:34-47) */
    /* tuning (ADMMSolverConfig) */
    float dt, g, mu, kappa, beta, thickness;
    int32_t admm_max_iter, dcd_interval, gs_max_iter, jacobi_iter;
    int32_t max_contacts;         /* contact slots (dcd.narrow.max_collision) */
    int32_t enable_contact, warmstart_ue, warmstart_uc;
    /* convergence control (no reference counterpart: the reference never
     * computes a residual, admm_impl_cpu.h:126,167).  residual_tol <= 0 runs
     * exactly admm_max_iter iterations like ADMMImplGPU::step. */
    float residual_tol;
    int32_t residual_check_every;
    /* BVH maintenance within a substep: 0 = full rebuild at every DCD (what
     * BVH_GPU::update does, collision_detection_cuda.cpp:126-144); 1 = rebuild at
     * the first DCD of a substep and refit the same tree at the later ones.  The
     * contact set does not depend on the tree, only the traversal cost does. */
    int32_t bvh_refit;
    /* Lanes per row of the sliced-ELL matrices (1, 2, 4 or 8); 0 = chosen by the
     * autotuner at create (cached per process and matrix shape, so handles of the
     * same scene sum in the same order). */
    int32_t ell_lanes;
    /* How the global step runs: 0 = chosen by the autotuner at create; 1 = one
     * kernel for the right-hand side and one per Jacobi sweep; 2 = one persistent
     * kernel for the right-hand side and all sweeps, its blocks synchronised
     * through per-block sweep counters (falls back to 1 when the device cannot
     * hold all blocks at once or jacobi_iter < 2); 3 = two sweeps per launch,
     * one block per spatially compact tile of rows, the halo rows computed
     * into shared memory.  All give identical bits. */
    int32_t jacobi_mode;
    /* Broad phase of the DCD: 0 = default (2); 1 = LBVH (the reference's
     * structure, bvh_refit applies); 2 = uniform-grid spatial hash.  Both report
     * the same pair set; the order of the contact list differs. */
    int32_t broad_phase;
    /* Global step solver (no reference counterpart beyond 0): 0 = jacobi_iter
     * Jacobi sweeps (ADMMImplGPU); 1 = pcg_iter iterations of conjugate gradients
     * preconditioned by diag(A); 2 = the same with the per-vertex 3x3 blocks set
     * by admm_b200_set_preconditioner (diag(A) until then).  pcg_iter 0 =
     * max(1, jacobi_iter / 2): the same kernel count as the Jacobi sweeps.
     * 3 = the learned global step of admm_b200_set_learned (until that call: the
     * Jacobi sweep written as x + (b - A x) / a_ii), judged per solve and with the
     * plain Jacobi substep as its fallback. */
    int32_t global_solver;
    int32_t pcg_iter;
    /* Optional [n_vert] friction coefficient per vertex (NULL: mu for all).  A
     * contact uses the coefficient of its first vertex (in slot order) that is
     * dynamic.  No reference counterpart (the reference has one mu per scene);
     * used by batches of bodies with different materials. */
    const float*   vert_mu;
    /* Lanes per DCD query of the grid broad phase (8, 16 or 32); 0 = chosen at
     * create from the number of queries: 32 while 32 lanes per query fill at most
     * four waves of the device (a latency-bound detection), else 16 or 8 (a
     * throughput-bound one).  All give the same contact list. */
    int32_t query_lanes;
    /* Contact predicates: 0 = the GPU backend's (dcdPT / dcdEE of dist_g.cuh:
     * interior closest points only, 0 <= d < thickness); 1 = the CPU backend's
     * ProximalQuery (narrow_phase.cpp:192-469: no pair of two static elements,
     * point-triangle at any closest point with d <= thickness, edge-edge with
     * d < thickness unless both closest points are segment end points, closest
     * points by Eberly's queries of distPT.h / distEE.h).  1 uses the grid broad
     * phase whatever broad_phase says. */
    int32_t contact_semantics;
    /* Solver semantics: 0 = the GPU backend's (ADMMImplGPU, admm_impl_gpu.cu:256-344);
     * 1 = the CPU backend's (ADMMImplCPU::step_fast, admm_impl_cpu.cpp:264-359):
     * Rayleigh damping Damp = dt (damp_k_L sum_{tri, tet, bending rows} w D_r^T D_r +
     * damp_k_M M) added to A and b_ini = Damp x0 added to every right-hand side
     * (admm_impl_cpu.cpp:191,221,295,344), S_c without the GPU backend's per-vertex
     * contact counts (compute_Scc, admm_impl_cpu.cpp:361-380), the friction-cone
     * projection as serial Gauss-Seidel over the contact list in its order
     * (_project_feasible_plain, admm_impl_cpu.cpp:390-407), and contact_semantics 1.
     * The reference factorises the damped A exactly (SimplicialLLT,
     * linear_solver_cpu.h:16-23); here the global step is global_solver 1 (conjugate
     * gradients) with pcg_iter iterations, enough to converge.  ABI version 5. */
    int32_t backend_semantics;
    float damp_k_L, damp_k_M;     /* ADMMSolverConfig defaults 1e-4 and 0 (admm_config.h:52-53) */
} AdmmB200Desc;

/* Per-step statistics (superset of Solver::StepMetrics, solver.h:29-45). */
typedef struct AdmmStepStats {
    int64_t frame;
    double  step_ms;          /* host wall time of the step call             */
    int32_t n_contacts;       /* contacts of the last DCD of the step         */
    int32_t admm_iters;       /* ADMM iterations run                          */
    double  primal_residual;  /* FP64 reductions, see admm_b200_residuals     */
    double  dual_residual;
    int32_t status;           /* ADMM_OK or a warning code (overflow, ...)    */
    int32_t peak_contacts;
} AdmmStepStats;

/* --- lifecycle ----------------------------------------------------------- */

/* Replaces ADMMImplGPU::convert_constraint2device + init + precompute
 * (admm_impl_gpu.cu:61-254) and BVH_GPU::init (collision_detection_cuda.cpp:39-83). */
int  admm_b200_create(const AdmmB200Desc* desc, int device, AdmmB200** out);
/* Frees the handle and every device buffer it owns. */
void admm_b200_destroy(AdmmB200* h);
/* Human-readable text of a status code. */
const char* admm_b200_errstr(int code);
/* Text of the last error on this handle (CUDA error string, argument name). */
const char* admm_b200_last_error(const AdmmB200* h);

/* --- stepping (IADMMBackend::step, admm_backend.h:17; ADMMImplGPU::step, admm_impl_gpu.cu:256-344) --- */

/* Runs n_steps substeps on the handle's stream (graph-replayed after the first
 * call).  stats may be NULL; when given it receives the last step's numbers
 * (this synchronises the stream). */
int  admm_b200_step(AdmmB200* h, int n_steps, AdmmStepStats* stats);
/* Enqueue n_steps substeps without synchronising (no stats). */
int  admm_b200_step_async(AdmmB200* h, int n_steps);
/* Block until all work on the handle's stream is done. */
int  admm_b200_sync(AdmmB200* h);

/* --- state (Solver::getVertices/getVelocities, solver.h:120-138; ADMMImplGPU::reset, admm_impl_gpu.cu:151-155) --- */

int  admm_b200_set_state(AdmmB200* h, const float* x_rowmajor, const float* v_rowmajor, int n);
int  admm_b200_get_state(AdmmB200* h, float* x_rowmajor, float* v_rowmajor, int n);
/* Restores the creation state and zeroes both dual variables. */
int  admm_b200_reset(AdmmB200* h);
/* Device pointers of the handle's row-major float4 state (x, v), for callers
 * that keep data on the GPU; valid until destroy.  The rows are in the library's
 * vertex order (below), not necessarily the caller's. */
int  admm_b200_device_state(AdmmB200* h, void** x_float4, void** v_float4);
/* With ADMM_B200_RENUMBER=1 in the environment at create, the library stores the dynamic
 * vertices in the Morton order of their rest positions (spatially close vertices at close
 * indices, for meshes whose own numbering has no locality); by default, and always with
 * backend_semantics 1 (whose serial Gauss-Seidel follows the contact order), it keeps the
 * caller's order.  Every other entry point takes and returns per-vertex data and vertex
 * indices in the caller's order.  order[i] receives the caller's index of internal row i;
 * static vertices keep their indices.  No reference counterpart. */
int  admm_b200_vertex_order(AdmmB200* h, int32_t* order, int n);

/* --- scripted static meshes (ScriptAnimator, src/solver/animator.cpp:9-204; applied at the
 * start of every substep as ADMMImplGPU::step does, admm_impl_gpu.cu:265-270) ---
 * Vertices [v_begin, v_end) of one static mesh (all >= n_dyn) follow a track.  Tracks are
 * applied in the order they are attached (attach them in mesh-id order, as the reference's
 * std::map does) and share the reference's frame counter: every substep advances it by one,
 * and a rigid track by one more before it reads its frame.  A rigid track places the rest
 * positions at pos[f] + quat[f] * rest (quat as x, y, z, w); a point track at
 * translate + rot9 * (scale * points[f]) (rot9 row-major).  Velocities are (new - old) / dt,
 * zero once a track has run past its last frame (which it then holds).  Attaching (and
 * admm_b200_reset) restarts the counter and places the meshes at their first frame with zero
 * velocity, as ADMMImplGPU::init does.  A rigid track needs at least 3 frames. */
int  admm_b200_set_rigid_track(AdmmB200* h, int32_t v_begin, int32_t v_end, int32_t n_frames,
                               const float* pos3, const float* quat4_xyzw);
int  admm_b200_set_point_track(AdmmB200* h, int32_t v_begin, int32_t v_end, int32_t n_frames,
                               const float* points3, const float* rot9, const float* translate3, float scale);
int  admm_b200_clear_tracks(AdmmB200* h);

/* --- ADMM internals, for parity tests and the fused dual/local step --- */

#define ADMM_BUF_X        0  /* [n_vert]  current positions (x_curr)   */
#define ADMM_BUF_X0       1  /* [n_vert]  step-start positions          */
#define ADMM_BUF_V        2  /* [n_vert]  velocities                    */
#define ADMM_BUF_P        3  /* [n_vert]  contact velocities p          */
#define ADMM_BUF_UC       4  /* [n_dyn]   contact dual Uc               */
#define ADMM_BUF_UE       5  /* [n_rows]  elastic dual Ue               */
#define ADMM_BUF_Z        6  /* [n_rows]  prox output z                 */
#define ADMM_BUF_B        7  /* [n_dyn]   global-step right-hand side   */
#define ADMM_BUF_MXT      8  /* [n_vert]  M * x_tilde                   */
/* Copy one N x 3 buffer (row-major floats) between host and device. */
int  admm_b200_read_buffer(AdmmB200* h, int which, float* out_rowmajor, int n);
int  admm_b200_write_buffer(AdmmB200* h, int which, const float* in_rowmajor, int n);

/* One local step z = prox(D*x + Ue) on the current buffers
 * (LocalProjectorGPU::project_elastic -> ADMMImplGPU::do_project_elastic,
 * admm_impl_gpu.cu:52-59). */
int  admm_b200_local_step(AdmmB200* h);
/* The global step: b from z, Ue, p, Uc (admm_impl_gpu.cu:307-318), then
 * jacobi_iter Jacobi sweeps on A (cu_jacobi_global, jacobi_solver.cu:141-180). */
int  admm_b200_global_step(AdmmB200* h);
/* Only the Jacobi sweeps on the current b and x (LinearSolverGPU::solve). */
int  admm_b200_jacobi(AdmmB200* h, int sweeps);
/* Pre-integration (do_pre_integration, jacobi_solver.cu:183-233). */
int  admm_b200_pre_integration(AdmmB200* h);

/* The contact sub-problem on the last detection (ADMMImplGPU::compute_Scc +
 * project_feasible_parallel, admm_impl_gpu.cu:296-303 and contact_solver.cu:402-431):
 * p = (x - x0 + Uc)/h, warm start, gs_max_iter friction-cone projections. */
int  admm_b200_contact_step(AdmmB200* h);

/* --- collision detection (ICollisionDetector, src/contact/icollision_detector.h:19-47) --- */

/* LBVH build + DCD on the handle's current x (BVH_GPU::update(Real*) + dcd(),
 * collision_detection_cuda.cpp:126-154) followed by the contact conversion
 * (convert_DCD_info, contact_solver.cu:158-185).  *count receives the contact
 * count (may exceed max_contacts, in which case ADMM_ERR_CONTACT_OVERFLOW is
 * returned and only max_contacts are stored). */
int  admm_b200_detect(AdmmB200* h, int* count);
/* ICollisionDetector::detect(pos): upload host positions, then detect. */
int  admm_b200_detect_host(AdmmB200* h, const float* x_rowmajor, int n, int* count);
/* Contacts of the last detection: pairs (v,f0,f1,f2) for point-triangle or
 * (e0a,e0b,e1a,e1b) for edge-edge, like BVH_GPU::d_collisonPairs; optional
 * outputs may be NULL.  bary = float4 (contact_solver.cu:139-141), normal and
 * point = float3, gap = h_cN. */
int  admm_b200_contacts(AdmmB200* h, int32_t* pairs_int4, float* bary4, float* normal3,
                        float* point3, float* gap, int cap, int* count);
/* contact_count / max_slots / peak_contact_count / clear of ICollisionDetector. */
int  admm_b200_contact_count(AdmmB200* h, int* count);
int  admm_b200_max_slots(AdmmB200* h, int* slots);
int  admm_b200_peak_contact_count(AdmmB200* h, int* peak);
int  admm_b200_clear_contacts(AdmmB200* h);

/* --- residuals (no reference counterpart) ---
 * primal = sqrt(sum_rows |w (Dx - z)|^2 + sum_dyn |w_c (x - x0 - h p)|^2), FP64;
 * dual   = sqrt(sum_rows |w (z - z_prev)|^2 + ...), FP64 on the GPU. */
int  admm_b200_residuals(AdmmB200* h, double* primal, double* dual);

/* --- host-buffer stepping (the reference's per-step host sync,
 * ADMMImplGPU::step with sync_to_host, admm_impl_gpu.cu:337-340) ---
 * Copies x_in/v_in (row-major n x 3, pinned host memory for full speed; v_in
 * may be NULL = keep the device velocities) to the device, runs one substep and
 * copies the new positions and velocities back into x_out/v_out.  Synchronous. */
int  admm_b200_step_host(AdmmB200* h, const float* x_in, const float* v_in, float* x_out, float* v_out, int n);

/* --- timing --- */
/* Phases of a substep (for admm_b200_phase_times). */
#define ADMM_PHASE_PRE       0
#define ADMM_PHASE_DCD       1
#define ADMM_PHASE_LOCAL     2
#define ADMM_PHASE_CONTACT   3
#define ADMM_PHASE_RHS       4
#define ADMM_PHASE_JACOBI    5
#define ADMM_PHASE_RESIDUAL  6
#define ADMM_PHASE_FINAL     7
#define ADMM_NUM_PHASES      8
/* Kernel classes that a graph probe can time (admm_b200_set_probe). */
#define ADMM_KERNEL_NONE            0
#define ADMM_KERNEL_LOCAL           1
#define ADMM_KERNEL_JACOBI          2
#define ADMM_KERNEL_RHS             3
#define ADMM_KERNEL_CONTACT_DU      4
#define ADMM_KERNEL_CONTACT_GATHER  5
#define ADMM_KERNEL_DCD_VF          6
#define ADMM_KERNEL_DCD_EE          7
/* set_probe argument: events at every phase change of the substep graph (outside
 * a residual_tol loop body); admm_b200_phase_times then returns the device time
 * between changes per phase, launch gaps included. */
#define ADMM_PROBE_PHASES         100

/* Device time (CUDA events on the handle's stream) per substep of the last
 * admm_b200_step call. */
int  admm_b200_last_step_device_ms(AdmmB200* h, float* ms);
/* enabled = 1: later steps run eagerly (no graph) with one CUDA event pair per
 * kernel launch; admm_b200_phase_times returns the summed kernel time and the
 * launch count of each ADMM_PHASE_* since the last call (and resets them). */
int  admm_b200_set_profiling(AdmmB200* h, int enabled);
int  admm_b200_phase_times(AdmmB200* h, double* ms, int64_t* launches, int n_phases);
/* Capture CUDA event pairs into the step graph around the launches of one
 * ADMM_KERNEL_* class (the first 64 launches of a substep); after each
 * synchronous admm_b200_step the durations are accumulated, and
 * admm_b200_probe_time returns their mean (ms per launch) and count, then resets. */
int  admm_b200_set_probe(AdmmB200* h, int kernel_class);
int  admm_b200_probe_time(AdmmB200* h, double* mean_ms, int64_t* count);
/* Number of kernels one substep launches (for launch accounting).  With
 * residual_tol > 0 the count depends on the iterations run: it is the count of
 * the most recent substep (before the first one, of a substep of one chunk). */
int  admm_b200_kernels_per_step(AdmmB200* h, int* n);
/* Autotuner choices made at create: lanes per row of the sliced-ELL copies of
 * A (Jacobi) and h^2 D^T W^2 (right-hand side), and the measured ms per launch. */
int  admm_b200_tuning(AdmmB200* h, int* lanes_a, int* lanes_r, float* ms_a, float* ms_r);
/* Per-vertex 3x3 preconditioner blocks (row-major, 9 floats per dynamic
 * vertex) for global_solver 2, e.g. the output of the learned preconditioner.
 * No reference counterpart. */
int  admm_b200_set_preconditioner(AdmmB200* h, const float* blocks9, int nd);
/* --- learned global step (global_solver 3; an addition with no reference
 * counterpart).  Replaces the jacobi_iter sweeps of cu_jacobi_global
 * (jacobi_solver.cu:141-180, called from admm_impl_gpu.cu:364) by `sweeps`
 * second-order sweeps
 *     x_{k+1} = x_k + omega[k] m (b - A x_k) + beta[k] (x_k - x_{k-1})   (beta[0] ignored)
 * from the warm start x_0 = x + theta (x - x_last) (x: the iterate the global step
 * receives, x_last: the one the previous global step of the substep received; no
 * warm start in a substep's first global step).  m [nd] scales the residual per
 * dynamic vertex (NULL: 1 / a_ii), theta [nd] is the warm-start coefficient (NULL:
 * 0); both come from the learned network (parallel_admm_b200/gnn.py).  Every solve is
 * judged on the device: a solve whose |b - A x_K| exceeds |b - A x_0| (and 1e-5 |b|)
 * fails and is replaced by the plain one (x as received, then jacobi_iter Jacobi
 * sweeps), in a conditional node of the substep graph: no host synchronisation.
 * sweeps <= 32. */
int  admm_b200_set_learned(AdmmB200* h, int sweeps, const float* omega, const float* beta, const float* m,
                           const float* theta, int nd);
/* out4: substeps run with the learned step, solves replaced by the plain Jacobi
 * solve, learned solves judged, learned solves that failed (= out4[1]). */
int  admm_b200_learned_stats(AdmmB200* h, int64_t* out4);
/* Kernels the plain solve that replaces a failed learned solve launches (for launch
 * accounting: a substep launches kernels_per_step plus this many per replaced solve). */
int  admm_b200_kernels_fallback(AdmmB200* h, int* n);
/* Training data: runs one substep (eagerly, with the handle's global solver) and
 * copies out, for its global step number `iteration` (1 .. admm_max_iter - 1,
 * counted from 0 over the substep), the right-hand side b, the iterate x_cur the
 * step receives and the iterate x_last the previous global step received (host,
 * row-major nd x 3).  The substep counts as a step of the simulation. */
int  admm_b200_record_global(AdmmB200* h, int iteration, float* b, float* x_cur, float* x_last, int nd);
/* How the global step runs (jacobi_mode): persistent = 1 for the one-kernel
 * global step (blocks = its grid), 3 for two sweeps per launch over row tiles,
 * 0 for one kernel per sweep; the autotuner's ms per global step with one
 * kernel per sweep and with the persistent kernel (0 when not timed). */
int  admm_b200_global_mode(AdmmB200* h, int* persistent, int* blocks, float* ms_sweeps, float* ms_persist);

/* --- learned block preconditioner (an addition with no reference counterpart) ---
 * A 3-layer message-passing network (width 64) over the graph of the global
 * matrix A predicts per dynamic vertex a 3x3 SPD block B_i = L_i L_i^T / a_ii
 * for admm_b200_set_preconditioner (global_solver 2); o = 0 gives diag(A)^-1.
 * It is trained on residual samples r of A x = b with the loss
 * mean_k |A B r_k - r_k|^2 / |r_k|^2 by the kernels of gnn.cu (forward,
 * backward, Adam).  The graph is A's off-diagonal CSR (symmetric pattern,
 * sorted columns); node features [n x 6], edge features [nnz x 2] as described
 * in parallel_admm_b200/gnn.py; set_graph swaps the system and keeps the
 * parameters and the Adam state.  bf16 = 1 rounds the weights to BF16 in the
 * forward and input-gradient products (FP32 accumulation). */
typedef struct AdmmGnn AdmmGnn;
int  admm_gnn_create(int bf16, AdmmGnn** out);
int  admm_gnn_set_graph(AdmmGnn* g, int n, int n_edges, const int32_t* start, const int32_t* col, const float* val,
                        const float* adiag, const float* node_feat, const float* edge_feat);
void admm_gnn_destroy(AdmmGnn* g);
int  admm_gnn_num_params(void);
int  admm_gnn_set_params(AdmmGnn* g, const float* theta, int n_params);
int  admm_gnn_get_params(AdmmGnn* g, float* theta, int n_params);
int  admm_gnn_forward(AdmmGnn* g, float* blocks9);
int  admm_gnn_loss_grad(AdmmGnn* g, const float* residuals, int k, double* loss, float* grad);
int  admm_gnn_adam(AdmmGnn* g, float lr);
/* The network's outputs for the learned global step (global_solver 3): per vertex
 * m_i = trace(B_i) / 3 (the isotropic part of the block; A is isotropic) and the
 * warm-start coefficient theta_i = clamp(o_i6, -1, 1) (host, n each); an all-zero
 * head gives m = 1 / a_ii and theta = 0, the plain Jacobi sweep. */
int  admm_gnn_outputs(AdmmGnn* g, float* m, float* theta);
/* Parameter gradient of a loss from its gradients gm, gtheta (host, n each) with
 * respect to admm_gnn_outputs; grad (host, may be NULL) receives it and the next
 * admm_gnn_adam applies it. */
int  admm_gnn_backward(AdmmGnn* g, const float* gm, const float* gtheta, float* grad);

/* --- training of the learned global step (an addition with no reference counterpart) ---
 * A context over one system A (off-diagonal CSR with start[n] entries, and the
 * diagonal).  admm_learn_loss_grad runs K sweeps of the learned global step from
 * the warm start x_c + theta (x_c - x_l) on each of nsamp samples (b, x_c, x_l, x*:
 * host, nsamp x n x 3, x* the converged solution of A x = b) and returns the mean
 * of |x_K - x*|_A^2 / |x_c - x*|_A^2 (+ mu |b - A x_K|^2 / |b - A x_c|^2 after
 * admm_learn_set_residual_weight, mu = 0 by default) and its gradients with respect to
 * omega, beta (K each), m and theta (n each); any gradient pointer may be NULL.
 * admm_learn_solve: conjugate gradients (diag(A) preconditioner) from x (host, in
 * and out) until |r|_{D^-1} <= rel_tol |r_0|_{D^-1} or max_iter iterations. */
typedef struct AdmmLearn AdmmLearn;
int  admm_learn_create(int n, const int32_t* start, const int32_t* col, const float* val, const float* diag,
                       AdmmLearn** out);
void admm_learn_destroy(AdmmLearn* L);
int  admm_learn_loss_grad(AdmmLearn* L, int K, const float* omega, const float* beta, const float* m,
                          const float* theta, int nsamp, const float* b, const float* x_c, const float* x_l,
                          const float* x_star, double* loss, float* g_omega, float* g_beta, float* g_m,
                          float* g_theta);
int  admm_learn_solve(AdmmLearn* L, const float* b, float* x, double rel_tol, int max_iter, int* iters);
int  admm_learn_set_residual_weight(AdmmLearn* L, double mu);

/* The global-step matrix A of a handle: nnz of the off-diagonal part when start
 * is NULL, else its CSR (start[n_dyn+1], col, val) and diagonal (host). */
int  admm_b200_system(AdmmB200* h, int32_t* start, int32_t* col, float* val, float* diag);

/* --- allocation-free Jacobi solve (no counterpart in the reference) ---
 * For callers that cannot allocate device memory themselves or through a handle
 * (their memory is owned by their own pool allocator, or cudaMalloc's latency and
 * implicit synchronisation are not acceptable in their loop).  Runs `sweeps`
 * Jacobi sweeps x <- D^-1 (b - (A - D) x) on caller-owned device buffers:
 * A's off-diagonal part in CSR (row_start[n+1], cols, vals), its diagonal diag[n],
 * b, x_in and x_out row-major n x 3 floats (x_out may equal x_in), enqueued on
 * `stream` (a cudaStream_t; NULL = the default stream).  Allocates nothing: the
 * ping-pong buffers are a static device array of 2 x 262144 x 3 floats, so
 * n <= 262144 (larger n returns ADMM_ERR_INVALID).  All calls in a process share
 * that array: calls that overlap on the GPU race.  The array's device address is
 * looked up in the calling thread's current context on every call made outside
 * stream capture and remembered per context (so callers in their own driver-API
 * contexts, and calls after a cudaDeviceReset, get the right address); a call made
 * during capture uses the remembered address, so make one call in that context
 * before any capture (else ADMM_ERR_STATE).  An error already pending on the
 * calling thread is not cleared: the call returns ADMM_ERR_CUDA without launching. */
int  admm_b200_jacobi_noalloc(int n, const int32_t* row_start, const int32_t* cols, const float* vals,
                              const float* diag, const float* b, const float* x_in, float* x_out, int sweeps,
                              void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ADMM_B200_H */
