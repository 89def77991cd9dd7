// admm_b200.cu -- the C ABI of the B200 ADMM substep (include/admm_b200.h).
//
// One handle = one scene on one GPU, one CUDA stream, and one CUDA graph that
// holds a whole substep (pre-integration, admm_max_iter ADMM iterations with a
// DCD every dcd_interval iterations, the final dual update and the post
// process).  Replaces ADMMImplGPU::step (admm_impl_gpu.cu:256-344), which
// launches ~25 + 2*GS + J kernels per iteration from the host with device
// synchronisations and device-to-host copies inside the loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "admm_b200.h"
#include "animate.cuh"
#include "contact.cuh"
#include "grid.cuh"
#include "kernels.cuh"
#include "lbvh.cuh"
#include "learn.cuh"
#include "scan_sort.cuh"
#include "setup.hpp"

using namespace admm;

struct AdmmB200 {
    int device = 0;
    cudaStream_t stream = nullptr;
    DevScene s;
    std::vector<void*> allocs;
    std::string last_error;
    // scripted static meshes
    std::vector<TrackDev> tracks;   // host copies of the track records (device pointers inside)
    AnimDev anim;
    // scene scalars
    int admm_max_iter = 0, dcd_interval = 1, gs_iter = 0, jac_iter = 0;
    int tet_blocks = 0, tri_blocks = 0, bend_blocks = 0, pin_blocks = 0;
    int contact_grid = 1;
    int group_grid = 1;             // blocks of the kernels that walk the touched list in lane groups
    int pass_grid = 1;              // blocks of the fused projection passes (a warp per contact)
    int warp_grid = 1;              // blocks of the kernels that walk it one warp per vertex
    int* hist = nullptr;       // radix histograms
    int sort_max = 0;
    std::vector<float4> x_init, v_init;
    // graph
    cudaGraphExec_t step_exec = nullptr;
    int kernels_per_step = 0;
    int launch_counter = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    int64_t frame = 0;
    int peak = 0;
    bool detected = false;
    float residual_tol = 0.f;
    int residual_every = 0;
    bool warmstart_ue = true, warmstart_uc = true;
    bool bvh_refit = true;
    bool use_grid = true;           // broad phase: uniform grid (true) or LBVH
    int global_solver = 0;          // 0 Jacobi, 1 PCG diag(A), 2 PCG learned blocks
    int pcg_iter = 0;
    PcgDev pcg;
    float* pcg_blocks = nullptr;    // [9 nd] learned blocks (global_solver 2)
    // learned global step (global_solver 3)
    LearnDev learn;
    int learn_sweeps = 0;
    std::vector<float> learn_omega, learn_beta;
    int* fail_host = nullptr;       // pinned copy of learn.fail (eager substeps)
    int64_t learn_substeps = 0;
    int kernels_fallback = 0;       // kernels of the plain solve that replaces a failed learned one
    cudaStream_t if_stream = nullptr;  // capture of the bodies of the fallback IF nodes
    bool force_plain = false;       // enqueue the Jacobi global step whatever global_solver says
    // Vertex renumbering (ADMM_B200_RENUMBER=1): the library stores the dynamic vertices in
    // the Morton order of their rest positions (spatially close vertices at close indices,
    // for meshes whose own numbering has no locality); every entry point that takes or
    // returns per-vertex data or vertex indices maps between that order and the caller's.
    // perm[internal] = caller's index, iperm[caller's] = internal; empty = identity, the
    // default (a lattice numbering gives each warp of the sweeps contiguous neighbour rows,
    // which the Morton order breaks up) and always with the CPU backend's semantics, whose
    // serial Gauss-Seidel follows the contact order.
    std::vector<int> perm, iperm;
    int* d_perm = nullptr;
    HostCsr hostA_caller;           // the global matrix in the caller's order (admm_b200_system)
    // recording of one global step's inputs (admm_b200_record_global, eager substeps)
    int rec_target = -1, rec_count = 0;
    float4 *rec_b = nullptr, *rec_cur = nullptr, *rec_last = nullptr;
    int enqueue_rc = ADMM_OK;       // first error while enqueueing or capturing a substep
    float grid_cell_size = 0.f;
    int grid_buckets = 0;
    int query_lanes = 32;           // lanes per grid DCD query (8, 16, 32)
    bool pdl = true;                // programmatic dependent launch between the kernels of a substep
    cudaStream_t cstream = nullptr; // stream the enqueue helpers launch on (capture target)
    cudaStream_t side = nullptr;    // second branch of an ADMM iteration (local step)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool overlap = true;
    cudaStream_t body_stream = nullptr;
    int chunk = 0;                  // ADMM iterations between residual checks (residual_tol > 0)
    bool in_body = false;           // capturing the body of the conditional node (no event nodes allowed)
    int kernels_body = 0;           // kernels of one conditional-body chunk
    int last_iters = 0;             // ADMM iterations of the most recent substep
    // autotuner choices (lanes per row of the sliced-ELL matrices) and their times
    int tune_lanes_a = 1, tune_lanes_r = 1;
    float tune_ms_a = 0.f, tune_ms_r = 0.f;
    // global step: persistent kernel (RHS + all sweeps) or one kernel per sweep
    PersistPlan pp;
    bool persist_ok = false;        // plan built and all blocks fit on the device at once
    bool persist = false;           // chosen mode: persistent global step
    bool tiled = false;             // chosen mode: two sweeps per launch over row tiles
    TileSet ts;
    int tile_smem = 0;
    HostCsr hostA;                  // the global matrix on the host (admm_b200_system)
    std::vector<float> hostAdiag;
    float tune_ms_tiled = 0.f;
    float tune_ms_persist = 0.f, tune_ms_sweeps = 0.f;  // one global step, both modes
    // host-buffer stepping
    float* stage = nullptr;    // [6n] row-major x then v
    // profiling: eager launches with one event pair per launch, tagged by phase
    bool profiling = false;
    int phase = 0;
    std::vector<cudaEvent_t> prof_ev;
    std::vector<int> prof_phase;
    int prof_used = 0;
    double phase_ms[ADMM_NUM_PHASES] = {0};
    int64_t phase_launches[ADMM_NUM_PHASES] = {0};
    // probes: event pairs captured into the step graph around one kernel class
    int probe_kernel = 0;           // ADMM_KERNEL_* class, or ADMM_PROBE_PHASES
    std::vector<cudaEvent_t> pev;   // phase probes: one event at every phase change of the graph
    std::vector<int> pev_phase, pev_launch;
    int pev_used = 0;
    std::vector<cudaEvent_t> probe_ev;
    int probe_used = 0;
    double probe_ms = 0.0;
    int64_t probe_n = 0;
};

namespace {

const char* kErrStr[] = {"ok",
                         "invalid argument",
                         "CUDA error",
                         "out of device memory",
                         "contact overflow (more contacts than max_contacts)",
                         "BVH traversal stack overflow",
                         "non-finite value",
                         "residual tolerance not reached",
                         "no usable sm_100 device",
                         "call out of order",
                         "device-side wait timed out"};

int fail(AdmmB200* h, int code, const std::string& what) {
    if (h) h->last_error = what;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            return fail(h, e_ == cudaErrorMemoryAllocation ? ADMM_ERR_OOM : ADMM_ERR_CUDA,    \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                  \
        }                                                                                     \
    } while (0)

template <class T>
int dalloc(AdmmB200* h, T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return fail(h, ADMM_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    h->allocs.push_back((void*)*p);
    e = cudaMemset(*p, 0, count * sizeof(T));
    if (e != cudaSuccess) return fail(h, ADMM_ERR_CUDA, cudaGetErrorString(e));
    return ADMM_OK;
}

template <class T>
int dupload(AdmmB200* h, T** p, const T* src, size_t count) {
    int rc = dalloc(h, p, count);
    if (rc) return rc;
    if (count && src) {
        cudaError_t e = cudaMemcpy(*p, src, count * sizeof(T), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return fail(h, ADMM_ERR_CUDA, cudaGetErrorString(e));
    }
    return ADMM_OK;
}

template <class T>
void dfree(AdmmB200* h, T* p) {
    if (!p) return;
    for (auto& a : h->allocs)
        if (a == (void*)p) {
            cudaFree(a);
            a = nullptr;
        }
}

#define TRY(x)                 \
    do {                       \
        int r_ = (x);          \
        if (r_) return r_;     \
    } while (0)

inline int blocks(int n, int t) { return n <= 0 ? 1 : (n + t - 1) / t; }

int alloc_bvh(AdmmB200* h, BvhDev& t, int n) {
    t.n = n;
    const int nn = n > 0 ? 2 * n - 1 : 1;
    TRY(dalloc(h, &t.box_lo, nn));
    TRY(dalloc(h, &t.box_up, nn));
    TRY(dalloc(h, &t.left, n));
    TRY(dalloc(h, &t.right, n));
    TRY(dalloc(h, &t.parent, nn));
    TRY(dalloc(h, &t.leaf_elem, n));
    TRY(dalloc(h, &t.flags, n));
    TRY(dalloc(h, &t.keys, n));
    TRY(dalloc(h, &t.keys_alt, n));
    TRY(dalloc(h, &t.vals, n));
    TRY(dalloc(h, &t.vals_alt, n));
    TRY(dalloc(h, &t.elem_lo, n));
    TRY(dalloc(h, &t.elem_up, n));
    TRY(dalloc(h, &t.scene, 8));
    TRY(dalloc(h, &t.node4, n > 1 ? 4 * (size_t)(n - 1) : 4));
    return ADMM_OK;
}

// ------------------------------ enqueue helpers -----------------------------
constexpr int kMaxProfEvents = 1 << 14;
constexpr int kMaxProbes = 64;

// Event bookkeeping around one launch: profiling (eager) and graph probes.
struct LaunchTimer {
    AdmmB200* h;
    int probe_id;
    cudaEvent_t a = nullptr, b = nullptr;
    bool prof = false, probe = false;
    LaunchTimer(AdmmB200* hh, int pid) : h(hh), probe_id(pid) {
        if (h->profiling && h->prof_used + 2 <= (int)h->prof_ev.size()) {
            prof = true;
            a = h->prof_ev[h->prof_used];
            b = h->prof_ev[h->prof_used + 1];
            h->prof_phase[h->prof_used / 2] = h->phase;
            h->prof_used += 2;
        } else if (!h->profiling && !h->in_body && pid != 0 && pid == h->probe_kernel &&
                   h->probe_used + 2 <= (int)h->probe_ev.size()) {
            probe = true;
            a = h->probe_ev[h->probe_used];
            b = h->probe_ev[h->probe_used + 1];
            h->probe_used += 2;
        }
        // inside stream capture only an external record becomes a timing node of the graph
        if (a) cudaEventRecordWithFlags(a, h->cstream, probe ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
    ~LaunchTimer() {
        if (b) cudaEventRecordWithFlags(b, h->cstream, probe ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
};

constexpr int kMaxPhaseEvents = 1024;

// Tags the launches that follow with phase `ph`.  With phase probes on, every
// phase change outside the conditional body also records an event into the
// graph, so that the device time between changes is charged to the phase.
void set_phase(AdmmB200* h, int ph) {
    if (h->probe_kernel == ADMM_PROBE_PHASES && !h->profiling && !h->in_body && ph != h->phase &&
        h->pev_used < (int)h->pev.size()) {
        cudaEventRecordWithFlags(h->pev[h->pev_used], h->cstream, cudaEventRecordExternal);
        h->pev_phase[h->pev_used] = ph;
        h->pev_launch[h->pev_used] = h->launch_counter;
        h->pev_used++;
    }
    h->phase = ph;
}

#define LAUNCH_P(pid, kernel, grid, block, ...)                                      \
    do {                                                                             \
        LaunchTimer lt_(h, (pid));                                                   \
        launch_k(kernel, dim3(grid), dim3(block), 0, h->cstream, h->pdl, __VA_ARGS__); \
        h->launch_counter++;                                                         \
    } while (0)
#define LAUNCH(kernel, grid, block, ...) LAUNCH_P(0, kernel, grid, block, __VA_ARGS__)
#define LAUNCH_SMEM(pid, kernel, grid, block, smem, ...)                                  \
    do {                                                                                 \
        LaunchTimer lt_(h, (pid));                                                       \
        launch_k(kernel, dim3(grid), dim3(block), smem, h->cstream, h->pdl, __VA_ARGS__); \
        h->launch_counter++;                                                             \
    } while (0)

void enqueue_refit(AdmmB200* h, BvhDev& t, const int* elems, int stride, bool tri) {
    const int n = t.n;
    if (n <= 0) return;
    if (tri) LAUNCH(k_leaf_refresh<3>, blocks(n, 256), 256, h->s.x, elems, stride, t);
    else LAUNCH(k_leaf_refresh<2>, blocks(n, 256), 256, h->s.x, elems, stride, t);
    LAUNCH(k_refit, blocks(n, 256), 256, t);
}

void enqueue_build(AdmmB200* h, BvhDev& t, const int* elems, int stride, bool tri) {
    const int n = t.n;
    if (n <= 0) return;
    if (tri) LAUNCH(k_elem_boxes<3>, blocks(n, 256), 256, h->s.x, elems, stride, n, t);
    else LAUNCH(k_elem_boxes<2>, blocks(n, 256), 256, h->s.x, elems, stride, n, t);
    LAUNCH(k_morton, blocks(n, 256), 256, t);
    if (n > 1) {
        LaunchTimer lt(h, 0);  // one timer around the 40 launches of the sort
        radix_sort(t.keys, t.vals, t.keys_alt, t.vals_alt, n, 64, h->hist, h->s.scan_tmp, h->cstream, h->pdl);
        h->launch_counter += 8 * 5;
    }
    LAUNCH(k_karras, blocks(n, 256), 256, t);
    LAUNCH(k_refit, blocks(n, 256), 256, t);
}

// Grid queries with h->query_lanes lanes per query (count or write pass).
void launch_grid_query(AdmmB200* h, bool write, int nq) {
    DevScene& s = h->s;
    const int g = blocks((int)std::min<int64_t>((int64_t)nq * h->query_lanes, INT32_MAX), kQueryThreads);
    switch (h->query_lanes * 2 + (write ? 1 : 0)) {
        case 16: LAUNCH(k_grid_count8, g, kQueryThreads, s); break;
        case 17: LAUNCH_P(ADMM_KERNEL_DCD_VF, (k_grid_query<true, 8>), g, kQueryThreads, s); break;
        case 32: LAUNCH((k_grid_query<false, 16>), g, kQueryThreads, s); break;
        case 33: LAUNCH_P(ADMM_KERNEL_DCD_VF, (k_grid_query<true, 16>), g, kQueryThreads, s); break;
        case 64: LAUNCH((k_grid_query<false, 32>), g, kQueryThreads, s); break;
        default: LAUNCH_P(ADMM_KERNEL_DCD_VF, (k_grid_query<true, 32>), g, kQueryThreads, s); break;
    }
}

// DCD + contact conversion + incidence lists + S_c / Gamma / K_c, all on device.
// rebuild = false refits the trees of the previous build.
void enqueue_dcd(AdmmB200* h, bool rebuild = true) {
    DevScene& s = h->s;
    set_phase(h, ADMM_PHASE_DCD);
    const int nq = s.nsv + s.nse;
    if (h->use_grid) {
        const int ne = s.nst + s.nse;
        cudaMemsetAsync(s.grid.ctr, 0, sizeof(int) * 4, h->cstream);
        if (ne > 0) {
            LAUNCH(k_grid_count, blocks(ne, 256), 256, s);
            {
                LaunchTimer lt(h, 0);
                exclusive_scan(s.grid.cnt, s.grid.start, h->grid_buckets, s.scan_tmp, s.grid.start + h->grid_buckets,
                               h->cstream, h->pdl);
                h->launch_counter += 3;
            }
            LAUNCH(k_grid_scatter, blocks(ne, 256), 256, s);
        }
        if (nq > 0) launch_grid_query(h, false, nq);
    } else {
        if (rebuild) {
            LAUNCH(k_scene_init, 1, 32, s.bf, s.be);
            enqueue_build(h, s.bf, (const int*)s.st, 4, true);
            enqueue_build(h, s.be, (const int*)s.se, 2, false);
        } else {
            enqueue_refit(h, s.bf, (const int*)s.st, 4, true);
            enqueue_refit(h, s.be, (const int*)s.se, 2, false);
        }
        if (s.nsv > 0) LAUNCH(k_dcd_vf<false>, blocks(s.nsv, 128), 128, s);
        if (s.nse > 0) LAUNCH(k_dcd_ee<false>, blocks(s.nse, 128), 128, s);
    }
    if (nq > 0) {
        LaunchTimer lt(h, 0);
        exclusive_scan(s.qcount, s.qoff, nq, s.scan_tmp, s.nc_raw, h->cstream, h->pdl);
        h->launch_counter += 3;
    } else {
        cudaMemsetAsync(s.nc_raw, 0, sizeof(int), h->cstream);
    }
    LAUNCH(k_set_count, 1, 1, s);
    if (h->use_grid) {
        if (nq > 0) launch_grid_query(h, true, nq);
    } else {
        if (s.nsv > 0) LAUNCH_P(ADMM_KERNEL_DCD_VF, k_dcd_vf<true>, blocks(s.nsv, 128), 128, s);
        if (s.nse > 0) LAUNCH_P(ADMM_KERNEL_DCD_EE, k_dcd_ee<true>, blocks(s.nse, 128), 128, s);
    }
    cudaMemsetAsync(s.vcnt, 0, sizeof(int) * s.n, h->cstream);
    cudaMemsetAsync(s.vfill, 0, sizeof(int) * s.n, h->cstream);
    LAUNCH(k_contact_count, h->contact_grid, kContactThreads, s);
    {
        LaunchTimer lt(h, 0);
        exclusive_scan(s.vcnt, s.vstart, s.n, s.scan_tmp, s.vstart + s.n, h->cstream, h->pdl);
        h->launch_counter += 3;
    }
    {
        LaunchTimer lt(h, 0);
        exclusive_scan(s.vcnt, s.tpos, s.n, s.scan_tmp, s.ntv, h->cstream, h->pdl, true);
        h->launch_counter += 3;
    }
    LAUNCH(k_contact_touched, blocks(s.n, kContactThreads), kContactThreads, s);
    LAUNCH(k_contact_fill, h->contact_grid, kContactThreads, s);
    LAUNCH(k_contact_sort_lists, h->warp_grid, kContactThreads, s);
    LAUNCH(k_contact_scc, h->contact_grid, kContactThreads, s);
    LAUNCH(k_contact_incidence, h->contact_grid, kContactThreads, s);
}

void enqueue_local(AdmmB200* h, int mode) {
    const int g = h->tet_blocks + h->tri_blocks + h->bend_blocks + h->pin_blocks;
    set_phase(h, ADMM_PHASE_LOCAL);
    if (mode == LOCAL_PROX)
        LAUNCH_P(ADMM_KERNEL_LOCAL, k_local<LOCAL_PROX>, g, kLocalThreads, h->s, h->tet_blocks, h->tri_blocks, h->bend_blocks);
    else if (mode == (LOCAL_PROX | LOCAL_DUAL))
        LAUNCH_P(ADMM_KERNEL_LOCAL, k_local<LOCAL_PROX | LOCAL_DUAL>, g, kLocalThreads, h->s, h->tet_blocks, h->tri_blocks,
                 h->bend_blocks);
    else
        LAUNCH(k_local<LOCAL_DUAL>, g, kLocalThreads, h->s, h->tet_blocks, h->tri_blocks, h->bend_blocks);
}

// Contact step of one ADMM iteration (project_impl, contact_solver.cu:316-431):
// p with the warm start, then gs_iter passes of friction-cone projection and
// gather.
int enqueue_contact(AdmmB200* h, bool dual) {
    DevScene& s = h->s;
    set_phase(h, ADMM_PHASE_CONTACT);
    const int split = blocks(s.nd, kVertThreads);
    if (dual) LAUNCH(k_contact_p<true>, split + h->group_grid, kVertThreads, s, split);
    else LAUNCH(k_contact_p<false>, split + h->group_grid, kVertThreads, s, split);
    const int G = h->gs_iter;
    if (G <= 0) return ADMM_OK;
    if (s.cpu_backend) {
        LAUNCH_P(ADMM_KERNEL_CONTACT_DU, k_contact_gs_serial, 1, 32, s, G);
        return ADMM_OK;
    }
    // pass 1 projects from s.p into s.du; pass g = 2..G rebuilds p of pass g-1
    // (P[g-1]) from P[g-2] and D[g-1] and projects into D[g]; the last gather
    // writes P[G] into s.p.  P[j] = s.p for even j, s.p2 for odd j; D[j] = s.du
    // for odd j, s.du2 for even j.
    auto P = [&](int j) { return (j & 1) ? s.p2 : s.p; };
    auto D = [&](int j) { return (j & 1) ? s.du : s.du2; };
    // k_contact_du, the passes and the last gather load detection data before their
    // dependency wait; that is legal only because the kernel launched right before each of
    // them (k_contact_p, then each pass) waits before it triggers (ADMM_PDL_WAIT_THEN_TRIGGER)
    // -- keep k_contact_p directly before this launch.
    LAUNCH_P(ADMM_KERNEL_CONTACT_DU, k_contact_du, h->contact_grid, kContactThreads, s);
    for (int g = 2; g <= G; g++)
        LAUNCH_P(ADMM_KERNEL_CONTACT_DU, k_contact_pass, h->pass_grid, kContactThreads, s, P(g - 2), P(g - 1),
                 D(g - 1), D(g));
    LAUNCH_P(ADMM_KERNEL_CONTACT_GATHER, k_contact_gather, h->group_grid, kContactThreads, s, P(G - 1), D(G));
    return ADMM_OK;
}

// one Jacobi sweep with the tuned number of lanes per row
void launch_jacobi(AdmmB200* h, const float4* src, float4* dst) {
    DevScene& s = h->s;
    const int g = blocks(s.A.nslices * 32, kVertThreads);
    switch (s.A.lanes) {
        case 1: LAUNCH_P(ADMM_KERNEL_JACOBI, k_jacobi<1>, g, kVertThreads, s, src, dst); break;
        case 2: LAUNCH_P(ADMM_KERNEL_JACOBI, k_jacobi<2>, g, kVertThreads, s, src, dst); break;
        case 4: LAUNCH_P(ADMM_KERNEL_JACOBI, k_jacobi<4>, g, kVertThreads, s, src, dst); break;
        default: LAUNCH_P(ADMM_KERNEL_JACOBI, k_jacobi<8>, g, kVertThreads, s, src, dst); break;
    }
}

void launch_jacobi2(AdmmB200* h, const float4* src, float4* dst) {
    DevScene& s = h->s;
    const size_t sm = (size_t)h->tile_smem;
    switch (s.A.lanes) {
        case 1: LAUNCH_SMEM(ADMM_KERNEL_JACOBI, k_jacobi2<1>, h->ts.ntiles, kTileThreads, sm, s, h->ts, src, dst); break;
        case 2: LAUNCH_SMEM(ADMM_KERNEL_JACOBI, k_jacobi2<2>, h->ts.ntiles, kTileThreads, sm, s, h->ts, src, dst); break;
        case 4: LAUNCH_SMEM(ADMM_KERNEL_JACOBI, k_jacobi2<4>, h->ts.ntiles, kTileThreads, sm, s, h->ts, src, dst); break;
        default: LAUNCH_SMEM(ADMM_KERNEL_JACOBI, k_jacobi2<8>, h->ts.ntiles, kTileThreads, sm, s, h->ts, src, dst); break;
    }
}

void launch_rhs(AdmmB200* h, bool save_prev) {
    DevScene& s = h->s;
    const int g = blocks(s.R.nslices * 32, kVertThreads);
#define RHS_CASE(T)                                                                          \
    if (save_prev) LAUNCH_P(ADMM_KERNEL_RHS, (k_rhs<T, true>), g, kVertThreads, s);          \
    else LAUNCH_P(ADMM_KERNEL_RHS, (k_rhs<T, false>), g, kVertThreads, s);
    switch (s.R.lanes) {
        case 1: RHS_CASE(1) break;
        case 2: RHS_CASE(2) break;
        case 4: RHS_CASE(4) break;
        default: RHS_CASE(8) break;
    }
#undef RHS_CASE
}

// The persistent global step: RHS (when rhs) and `sweeps` >= 2 Jacobi sweeps in
// one cooperative launch, no programmatic early start (its blocks spin).
void launch_persist(AdmmB200* h, bool rhs, bool save_prev, int sweeps) {
    DevScene& s = h->s;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(h->pp.blocks);
    cfg.blockDim = dim3(kPersistThreads);
    cfg.stream = h->cstream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    LaunchTimer lt_(h, ADMM_KERNEL_JACOBI);
    void (*k)(DevScene, PersistPlan, int) = nullptr;
#define PERSIST_R(T, TR)                                              \
    k = !rhs ? k_global_persist<T, TR, false, false>                  \
        : save_prev ? k_global_persist<T, TR, true, true>             \
                    : k_global_persist<T, TR, true, false>;
#define PERSIST_A(T)                                   \
    switch (s.R.lanes) {                               \
        case 1: PERSIST_R(T, 1) break;                 \
        case 2: PERSIST_R(T, 2) break;                 \
        case 4: PERSIST_R(T, 4) break;                 \
        default: PERSIST_R(T, 8) break;                \
    }
    switch (s.A.lanes) {
        case 1: PERSIST_A(1) break;
        case 2: PERSIST_A(2) break;
        case 4: PERSIST_A(4) break;
        default: PERSIST_A(8) break;
    }
#undef PERSIST_A
#undef PERSIST_R
    cudaLaunchKernelEx(&cfg, k, s, h->pp, sweeps);
    h->launch_counter++;
}

void enqueue_jacobi(AdmmB200* h, int sweeps) {
    DevScene& s = h->s;
    const int vb = blocks(s.nd, kVertThreads);
    set_phase(h, ADMM_PHASE_JACOBI);
    if (sweeps <= 0) return;
    if (h->persist && sweeps >= 2) {
        launch_persist(h, false, false, sweeps);
        return;
    }
    if (sweeps == 1) {
        launch_jacobi(h, s.x, s.jac[0]);
        LAUNCH(k_copy_dyn, vb, kVertThreads, s, s.jac[0], s.x);
        return;
    }
    if (h->tiled) {
        // pairs of sweeps x -> jac0 -> jac1 -> ...; the last pair writes x when its
        // source is not x, an odd sweep count ends with one plain sweep into x
        const int pairs = sweeps / 2, odd = sweeps & 1;
        const float4* src = s.x;
        for (int p = 0; p < pairs; p++) {
            float4* dst = (p == pairs - 1 && !odd && src != s.x) ? s.x : s.jac[p & 1];
            launch_jacobi2(h, src, dst);
            src = dst;
        }
        if (odd) launch_jacobi(h, src, s.x);
        else if (src != s.x) LAUNCH(k_copy_dyn, vb, kVertThreads, s, src, s.x);
        return;
    }
    for (int k = 0; k < sweeps; k++) {
        const float4* src = k == 0 ? s.x : s.jac[(k - 1) & 1];
        float4* dst = k == sweeps - 1 ? s.x : s.jac[k & 1];
        launch_jacobi(h, src, dst);
    }
}

// PCG global step: init, then `iters` updates with an A u product between them
// (2 iters + 1 launches); the result is in x.
void enqueue_pcg(AdmmB200* h, int iters) {
    DevScene& s = h->s;
    set_phase(h, ADMM_PHASE_JACOBI);
    if (iters <= 0 || s.nd <= 0) return;
    const int ga = blocks(s.A.nslices * 32, kVertThreads), gv = blocks(s.nd, kVertThreads);
    PcgDev& g = h->pcg;
    g.block = (h->global_solver == 2 && h->pcg_blocks) ? h->pcg_blocks : nullptr;
#define PCG_T(T)                                                                        \
    do {                                                                                \
        LAUNCH(k_pcg_init<T>, ga, kVertThreads, s, g);                                  \
        LAUNCH(k_pcg_spmv<T>, ga, kVertThreads, s, g);                                  \
        for (int it = 0; it < iters; it++) {                                            \
            LAUNCH_P(ADMM_KERNEL_JACOBI, k_pcg_update, gv, kVertThreads, s, g, it);     \
            if (it + 1 < iters) LAUNCH(k_pcg_spmv<T>, ga, kVertThreads, s, g);          \
        }                                                                               \
    } while (0)
    switch (s.A.lanes) {
        case 1: PCG_T(1); break;
        case 2: PCG_T(2); break;
        case 4: PCG_T(4); break;
        default: PCG_T(8); break;
    }
#undef PCG_T
}

// The judge's pass over x (k_ljudge, lanes of A).
void launch_ljudge(AdmmB200* h) {
    DevScene& s = h->s;
    LearnDev& L = h->learn;
    switch (s.A.lanes) {
        case 1: LAUNCH(k_ljudge<1>, L.blocks, kVertThreads, s, L); break;
        case 2: LAUNCH(k_ljudge<2>, L.blocks, kVertThreads, s, L); break;
        case 4: LAUNCH(k_ljudge<4>, L.blocks, kVertThreads, s, L); break;
        default: LAUNCH(k_ljudge<8>, L.blocks, kVertThreads, s, L); break;
    }
}

// The plain solve that replaces a failed learned one: x <- x as received (L.xl), the
// jacobi_iter Jacobi sweeps on the same b, and the judge's pass to refresh A x for the
// next global step.
void enqueue_learned_replacement(AdmmB200* h) {
    DevScene& s = h->s;
    LAUNCH(k_copy_dyn, blocks(s.nd, kVertThreads), kVertThreads, s, (const float4*)h->learn.xl, s.x);
    enqueue_jacobi(h, h->jac_iter);
    launch_ljudge(h);
}

// The decision on a learned solve and the plain solve that replaces a failed one.  In a
// graph the replacement is the body of an IF node after k_ldecide, which sets its
// condition (inside the residual-tolerance WHILE body the IF node is nested in it);
// eagerly, the host reads the decision (one stream synchronisation per solve).
void enqueue_learned_decide(AdmmB200* h, bool first) {
    LearnDev& L = h->learn;
    const int fi = first ? 1 : 0;
    cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamGetCaptureInfo(h->cstream, &cst, nullptr, &g, nullptr, nullptr);
    if (e != cudaSuccess) {
        if (h->enqueue_rc == ADMM_OK) h->enqueue_rc = fail(h, ADMM_ERR_CUDA, cudaGetErrorString(e));
        return;
    }
    if (cst != cudaStreamCaptureStatusActive) {
        LAUNCH(k_ldecide, 1, kDecideThreads, L, cudaGraphConditionalHandle(0), 0, fi);
        int failed = 0;
        if (cudaMemcpyAsync(h->fail_host, L.fail, sizeof(int), cudaMemcpyDeviceToHost, h->cstream) == cudaSuccess &&
            cudaStreamSynchronize(h->cstream) == cudaSuccess)
            failed = *h->fail_host;
        if (failed) enqueue_learned_replacement(h);
        return;
    }
    cudaGraphConditionalHandle cond;
    e = cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault);
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    if (e == cudaSuccess) {
        LAUNCH(k_ldecide, 1, kDecideThreads, L, cond, 1, fi);
        e = cudaStreamGetCaptureInfo(h->cstream, &cst, nullptr, &g, &deps, &ndeps);
    }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
    if (e != cudaSuccess) {
        if (h->enqueue_rc == ADMM_OK) h->enqueue_rc = fail(h, ADMM_ERR_CUDA, std::string("fallback IF node: ") + cudaGetErrorString(e));
        return;
    }
    cudaStream_t parent = h->cstream;
    const bool was_in_body = h->in_body;
    const int before = h->launch_counter;
    h->cstream = h->if_stream;
    h->in_body = true;
    e = cudaStreamBeginCaptureToGraph(h->cstream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_learned_replacement(h);
        cudaGraph_t bg = nullptr;
        e = cudaStreamEndCapture(h->cstream, &bg);
    }
    h->kernels_fallback = h->launch_counter - before;
    h->launch_counter = before;
    h->in_body = was_in_body;
    h->cstream = parent;
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(h->cstream, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess && h->enqueue_rc == ADMM_OK)
        h->enqueue_rc = fail(h, ADMM_ERR_CUDA, std::string("fallback IF body: ") + cudaGetErrorString(e));
}

// The learned global step: right-hand side with the start of the solve, learn_sweeps
// second-order sweeps (x_k in {x, jac0, jac1}[(s0 + k) % 3], s0 = -K mod 3, so that x_K
// lands in x), the judge's pass and the decision with its fallback.
void enqueue_learned(AdmmB200* h, bool save_prev, bool first) {
    DevScene& s = h->s;
    LearnDev& L = h->learn;
    const int K = h->learn_sweeps;
    const int s0 = (3 - K % 3) % 3;
    float4* buf[3] = {s.x, s.jac[0], s.jac[1]};
    set_phase(h, ADMM_PHASE_RHS);
    const int ex = first ? 0 : 1;
#define RHSL_CASE(T)                                                                                             \
    if (save_prev) LAUNCH_P(ADMM_KERNEL_RHS, (k_rhs_learn<T, true>), L.rblocks, kVertThreads, s, L, ex, buf[s0]); \
    else LAUNCH_P(ADMM_KERNEL_RHS, (k_rhs_learn<T, false>), L.rblocks, kVertThreads, s, L, ex, buf[s0]);
    switch (s.R.lanes) {
        case 1: RHSL_CASE(1) break;
        case 2: RHSL_CASE(2) break;
        case 4: RHSL_CASE(4) break;
        default: RHSL_CASE(8) break;
    }
#undef RHSL_CASE
    set_phase(h, ADMM_PHASE_JACOBI);
#define LS_CASE(T)                                                                                         \
    for (int k = 0; k < K; k++) {                                                                          \
        const float4* src = buf[(s0 + k) % 3];                                                             \
        const float4* prv = buf[(s0 + k + 2) % 3];                                                         \
        float4* dst = buf[(s0 + k + 1) % 3];                                                               \
        if (k == 0)                                                                                        \
            LAUNCH_P(ADMM_KERNEL_JACOBI, (k_lsweep<T, true>), L.blocks, kVertThreads, s, L, src, prv, dst, \
                     h->learn_omega[k], h->learn_beta[k], ex);                                             \
        else                                                                                               \
            LAUNCH_P(ADMM_KERNEL_JACOBI, (k_lsweep<T, false>), L.blocks, kVertThreads, s, L, src, prv, dst, \
                     h->learn_omega[k], h->learn_beta[k], 0);                                              \
    }
    switch (s.A.lanes) {
        case 1: LS_CASE(1) break;
        case 2: LS_CASE(2) break;
        case 4: LS_CASE(4) break;
        default: LS_CASE(8) break;
    }
#undef LS_CASE
    launch_ljudge(h);
    enqueue_learned_decide(h, first);
}

// Copies of one global step's inputs for admm_b200_record_global (eager only):
// x as received by global step rec_target - 1 and rec_target, b of rec_target.
void record_before_rhs(AdmmB200* h) {
    if (h->rec_target < 0) return;
    const size_t bytes = sizeof(float4) * (size_t)h->s.nd;
    if (h->rec_count == h->rec_target - 1) cudaMemcpyAsync(h->rec_last, h->s.x, bytes, cudaMemcpyDeviceToDevice, h->cstream);
    if (h->rec_count == h->rec_target) cudaMemcpyAsync(h->rec_cur, h->s.x, bytes, cudaMemcpyDeviceToDevice, h->cstream);
}

void record_after_rhs(AdmmB200* h) {
    if (h->rec_target < 0) return;
    if (h->rec_count == h->rec_target)
        cudaMemcpyAsync(h->rec_b, h->s.b, sizeof(float4) * (size_t)h->s.nd, cudaMemcpyDeviceToDevice, h->cstream);
    h->rec_count++;
}

void enqueue_global(AdmmB200* h, bool save_prev, bool first) {
    record_before_rhs(h);
    if (h->global_solver == 3 && !h->force_plain && h->rec_target < 0) {
        enqueue_learned(h, save_prev, first);
        record_after_rhs(h);
        return;
    }
    if (h->global_solver == 3 && !h->force_plain) {
        // recording: the right-hand side alone first, so that b can be copied
        // before the sweeps (the learned step then runs its own right-hand side)
        launch_rhs(h, false);
        record_after_rhs(h);
        enqueue_learned(h, save_prev, first);
        return;
    }
    if (h->global_solver > 0 && h->global_solver < 3) {
        set_phase(h, ADMM_PHASE_RHS);
        launch_rhs(h, save_prev);
        record_after_rhs(h);
        enqueue_pcg(h, h->pcg_iter);
        return;
    }
    if (h->persist && h->jac_iter >= 2 && h->rec_target < 0) {
        set_phase(h, ADMM_PHASE_JACOBI);
        launch_persist(h, true, save_prev, h->jac_iter);
        return;
    }
    set_phase(h, ADMM_PHASE_RHS);
    launch_rhs(h, save_prev);
    record_after_rhs(h);
    enqueue_jacobi(h, h->jac_iter);
}

// Persistent-kernel plan: rows in blocks of a multiple of 32 (at most one block
// per SM), and for each block the other blocks owning a column of its rows in
// the off-diagonal pattern of A, made symmetric.
int build_persist_plan(AdmmB200* h, const HostCsr& A) {
    DevScene& s = h->s;
    h->persist_ok = false;
    if (s.nd <= 0) return ADMM_OK;
    int sms = 0, coop = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device));
    if (!coop || sms <= 0) return ADMM_OK;
    const int groups = (s.nd + 31) / 32;
    const int per = (groups + sms - 1) / sms;
    const int rb = 32 * per;
    const int nb = (s.nd + rb - 1) / rb;
    std::vector<std::vector<int>> dep(nb);
    for (int i = 0; i < s.nd; i++) {
        const int gi = i / rb;
        for (int k = A.start[i]; k < A.start[i + 1]; k++) {
            const int gj = A.col[k] / rb;
            if (gj != gi) {
                dep[gi].push_back(gj);
                dep[gj].push_back(gi);
            }
        }
    }
    std::vector<int> ptr(nb + 1, 0), idx;
    for (int g = 0; g < nb; g++) {
        auto& v = dep[g];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        idx.insert(idx.end(), v.begin(), v.end());
        ptr[g + 1] = (int)idx.size();
    }
    int *dp = nullptr, *di = nullptr;
    unsigned* ep = nullptr;
    TRY(dupload(h, &dp, ptr.data(), ptr.size()));
    TRY(dupload(h, &di, idx.data(), idx.size()));
    TRY(dalloc(h, &ep, nb));
    h->pp.blocks = nb;
    h->pp.rows_per_block = rb;
    h->pp.dep_ptr = dp;
    h->pp.dep_idx = di;
    h->pp.epoch = ep;
    h->pp.spin_limit = 1 << 22;  // ~1-2 s of polling
    // every instantiation has the same launch bounds (kPersistThreads, 1 block per SM)
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_global_persist<8, 8, true, true>, kPersistThreads, 0));
    h->persist_ok = per_sm >= 1 && nb <= per_sm * sms;
    return ADMM_OK;
}

// Row tiles of the two-sweep kernel for the lanes A was tuned to, uploaded.
int upload_host_ell(AdmmB200* h, const HostEll& e, SlicedEll& out) {
    int *p = nullptr, *c = nullptr;
    float* v = nullptr;
    TRY(dupload(h, &p, e.ptr.data(), e.ptr.size()));
    TRY(dupload(h, &c, e.col.data(), e.col.size()));
    TRY(dupload(h, &v, e.val.data(), e.val.size()));
    out.rows = e.rows;
    out.nslices = e.nslices;
    out.lanes = e.lanes;
    out.ptr = p;
    out.col = c;
    out.val = v;
    return ADMM_OK;
}

int build_tiles_dev(AdmmB200* h, const HostCsr& A) {
    DevScene& s = h->s;
    if (s.nd <= 0) return ADMM_OK;
    std::vector<float> pos(3 * (size_t)s.nd);
    for (int i = 0; i < s.nd; i++) {
        pos[3 * i] = h->x_init[i].x;
        pos[3 * i + 1] = h->x_init[i].y;
        pos[3 * i + 2] = h->x_init[i].z;
    }
    const HostTiles t = build_tiles(A, s.nd, pos.data(), 3, kTileOwn, s.A.lanes);
    TileSet& d = h->ts;
    d.ntiles = t.ntiles;
    int* a;
    TRY(dupload(h, &a, t.row0.data(), t.row0.size())); d.row0 = a;
    TRY(dupload(h, &a, t.nlocal.data(), t.nlocal.size())); d.nlocal = a;
    TRY(dupload(h, &a, t.nown.data(), t.nown.size())); d.nown = a;
    TRY(dupload(h, &a, t.s1_0.data(), t.s1_0.size())); d.s1_0 = a;
    TRY(dupload(h, &a, t.s1_n.data(), t.s1_n.size())); d.s1_n = a;
    TRY(dupload(h, &a, t.s2_0.data(), t.s2_0.size())); d.s2_0 = a;
    TRY(dupload(h, &a, t.s2_n.data(), t.s2_n.size())); d.s2_n = a;
    TRY(dupload(h, &a, t.trow.data(), t.trow.size())); d.trow = a;
    TRY(upload_host_ell(h, t.e1, d.e1));
    TRY(upload_host_ell(h, t.e2, d.e2));
    h->tile_smem = (int)(sizeof(float4) * (size_t)std::max(t.max_local, 1));
    if (h->tile_smem > 48 * 1024) {
        const int lim = h->tile_smem;
        CK(cudaFuncSetAttribute(k_jacobi2<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_jacobi2<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_jacobi2<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(k_jacobi2<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    }
    return ADMM_OK;
}

// Milliseconds of one global step (RHS + jac_iter sweeps) in the given mode,
// timed as a captured graph of 8 global steps (as the substep graph runs them,
// with programmatic dependent launch); +inf when the mode cannot be captured.
int time_global(AdmmB200* h, int mode, float* ms) {
    const bool keep = h->persist, keep_t = h->tiled;
    h->persist = mode == 2;
    h->tiled = mode == 3;
    h->force_plain = true;
    h->cstream = h->stream;
    constexpr int kReps = 8;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    bool ok = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        for (int r = 0; r < kReps; r++) enqueue_global(h, false, false);
        ok = cudaStreamEndCapture(h->stream, &g) == cudaSuccess && g;
    }
    ok = ok && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    h->persist = keep;
    h->tiled = keep_t;
    h->force_plain = false;
    if (!ok) {
        cudaGetLastError();
        if (ge) cudaGraphExecDestroy(ge);
        *ms = 1e30f;
        return ADMM_OK;
    }
    CK(cudaGraphLaunch(ge, h->stream));  // warm-up
    CK(cudaEventRecord(h->ev0, h->stream));
    CK(cudaGraphLaunch(ge, h->stream));
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    cudaGraphExecDestroy(ge);
    CK(cudaGetLastError());
    int e[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(e, h->s.err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e[3]) return fail(h, ADMM_ERR_TIMEOUT, "persistent global step: a block wait timed out");
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    *ms = t / kReps;
    return ADMM_OK;
}

int upload_ell(AdmmB200* h, const HostCsr& c, int rows, int lanes, SlicedEll& out, HostEll* keep = nullptr) {
    HostEll e = csr_to_sliced_ell(c, rows, lanes, true);
    int *p = nullptr, *cc = nullptr, *rid = nullptr;
    float* v = nullptr;
    TRY(dupload(h, &p, e.ptr.data(), e.ptr.size()));
    TRY(dupload(h, &cc, e.col.data(), e.col.size()));
    TRY(dupload(h, &v, e.val.data(), e.val.size()));
    if (!e.rowid.empty()) TRY(dupload(h, &rid, e.rowid.data(), e.rowid.size()));
    out.rows = rows;
    out.nslices = e.nslices;
    out.lanes = lanes;
    out.ptr = p;
    out.col = cc;
    out.val = v;
    out.rowid = rid;
    if (keep) *keep = std::move(e);
    return ADMM_OK;
}

void free_ell(AdmmB200* h, SlicedEll& m) {
    dfree(h, const_cast<int*>(m.ptr));
    dfree(h, const_cast<int*>(m.col));
    dfree(h, const_cast<float*>(m.val));
    dfree(h, const_cast<int*>(m.rowid));
    m = SlicedEll{};
}

// Autotuner: lanes per row (1, 2, 4, 8) of both sliced-ELL matrices, chosen by
// timing 10 launches of each candidate on this device with this scene.  The
// choice is cached per (device, matrix shape) for the life of the process so
// that every handle of one scene sums in the same order; `fixed` > 0 skips the
// search and uses that many lanes.
struct TuneKey {
    int device, which, rows;
    int64_t nnz;
    bool operator==(const TuneKey& o) const {
        return device == o.device && which == o.which && rows == o.rows && nnz == o.nnz;
    }
};
std::mutex g_tune_mu;
std::vector<std::pair<TuneKey, std::pair<int, float>>> g_tune_cache;

// Device time of one Jacobi sweep (which = 0) or RHS launch (1) at the current
// lane count, as the step graph runs them: a graph of kTuneLaunches dependent
// launches (sweeps ping-pong between the two iterate buffers) with programmatic
// dependent launch between them, run once to warm up and then kTuneReps times;
// the fastest repetition counts.  Ten stream launches timed once ranked lane
// counts that lie within a few per cent of each other in the wrong order.
int time_ell(AdmmB200* h, int which, float* ms_per_launch) {
    constexpr int kTuneLaunches = 40, kTuneReps = 3;
    DevScene& s = h->s;
    const cudaStream_t keep = h->cstream;
    const int counter = h->launch_counter;
    h->cstream = h->stream;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int r = 0; r < kTuneLaunches; r++) {
        if (which == 0) launch_jacobi(h, r == 0 ? s.x : s.jac[(r + 1) & 1], s.jac[r & 1]);
        else launch_rhs(h, false);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
    h->cstream = keep;
    h->launch_counter = counter;
    CK(ce);
    cudaGraphExec_t ge = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    float best = 1e30f;
    cudaError_t e = cudaGraphLaunch(ge, h->stream);
    for (int k = 0; k < kTuneReps && e == cudaSuccess; k++) {
        e = cudaEventRecord(h->ev0, h->stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(ge, h->stream);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev1, h->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(h->ev1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        if (e == cudaSuccess) best = std::min(best, ms);
    }
    cudaGraphExecDestroy(ge);
    CK(e);
    CK(cudaGetLastError());
    *ms_per_launch = best / (float)kTuneLaunches;
    return ADMM_OK;
}

int autotune_ell(AdmmB200* h, const Assembly& as, int fixed, int* chosen_a, int* chosen_r, float* ms_a, float* ms_r) {
    DevScene& s = h->s;
    const int cand[4] = {1, 2, 4, 8};
    for (int which = 0; which < 2; which++) {
        const HostCsr& c = which == 0 ? as.A : as.R;
        SlicedEll& target = which == 0 ? s.A : s.R;
        const TuneKey key{h->device, which, s.nd, (int64_t)c.col.size()};
        int best_l = fixed;
        float best = 0.f;
        if (best_l == 0) {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            for (auto& e : g_tune_cache)
                if (e.first == key) {
                    best_l = e.second.first;
                    best = e.second.second;
                }
        }
        if (best_l == 0) {
            best = 1e30f;
            for (int k = 0; k < 4; k++) {
                TRY(upload_ell(h, c, s.nd, cand[k], target));
                float ms = 0.f;
                TRY(time_ell(h, which, &ms));
                free_ell(h, target);
                if (ms < best) {
                    best = ms;
                    best_l = cand[k];
                }
            }
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache.push_back({key, {best_l, best}});
        }
        TRY(upload_ell(h, c, s.nd, best_l, target));
        if (best == 0.f) TRY(time_ell(h, which, &best));
        if (which == 0) { *chosen_a = best_l; *ms_a = best; }
        else { *chosen_r = best_l; *ms_r = best; }
    }
    return ADMM_OK;
}

void enqueue_residual(AdmmB200* h) {
    DevScene& s = h->s;
    set_phase(h, ADMM_PHASE_RESIDUAL);
    const int vb = blocks(s.nd, kLocalThreads);
    const int g = h->tet_blocks + h->tri_blocks + h->bend_blocks + h->pin_blocks + vb;
    LAUNCH(k_residual, g, kLocalThreads, s, h->tet_blocks, h->tri_blocks, h->bend_blocks, h->pin_blocks);
    LAUNCH(k_residual_reduce, 1, 256, s, g);
}

// One ADMM iteration `it` of a substep (first: no dual update before it).  The
// BVH is built by the first detection of a substep (it == 0 of the first chunk)
// and refitted by the later ones unless bvh_refit is off.
void enqueue_iteration(AdmmB200* h, int it, bool first, bool residual) {
    DevScene& s = h->s;
    const int local_mode = first ? LOCAL_PROX : (LOCAL_PROX | LOCAL_DUAL);
    // The local step (z, Ue) and the detection + contact step (p, Uc) read x and
    // write disjoint data: with contact they run as two branches of the graph,
    // joined before the right-hand side.  Not inside the body of a conditional
    // node (iterations after the first chunk of a residual-tolerance substep),
    // whose capture keeps to one stream, and not under phase probes.
    const bool branches = s.contact && h->overlap && !h->in_body && h->probe_kernel != ADMM_PROBE_PHASES;
    cudaStream_t main = h->cstream;
    if (branches) {
        cudaEventRecord(h->ev_fork, main);
        cudaStreamWaitEvent(h->side, h->ev_fork, 0);
        h->cstream = h->side;
        enqueue_local(h, local_mode);
        cudaEventRecord(h->ev_join, h->side);
        h->cstream = main;
    } else {
        if (s.contact && it % h->dcd_interval == 0) enqueue_dcd(h, !h->bvh_refit || first);
        enqueue_local(h, local_mode);
    }
    if (branches && it % h->dcd_interval == 0) enqueue_dcd(h, !h->bvh_refit || first);
    if (s.contact) {
        const int rc = enqueue_contact(h, !first);
        if (rc != ADMM_OK && h->enqueue_rc == ADMM_OK) h->enqueue_rc = rc;
    }
    if (branches) cudaStreamWaitEvent(main, h->ev_join, 0);
    enqueue_global(h, residual, first);
    if (residual) enqueue_residual(h);
}

void enqueue_step_begin(AdmmB200* h) {
    DevScene& s = h->s;
    set_phase(h, ADMM_PHASE_PRE);
    if (h->anim.n_tracks > 0) {
        LAUNCH(k_anim_advance, 1, 32, h->anim, 0);
        LAUNCH(k_animate, blocks(h->anim.n_verts, kVertThreads), kVertThreads, s, h->anim);
    }
    LAUNCH(k_pre_integration, blocks(s.n, kVertThreads), kVertThreads, s);
    if (s.cpu_backend) LAUNCH(k_damp_binit, blocks(s.nd, kVertThreads), kVertThreads, s);
    if (!h->warmstart_ue) cudaMemsetAsync(s.ue, 0, sizeof(float4) * s.m, h->cstream);
    if (!h->warmstart_uc) cudaMemsetAsync(s.uc, 0, sizeof(float4) * s.nd, h->cstream);
}

void enqueue_step_end(AdmmB200* h) {
    DevScene& s = h->s;
    enqueue_local(h, LOCAL_DUAL);
    set_phase(h, ADMM_PHASE_FINAL);
    LAUNCH(k_vertex_final, blocks(s.n, kVertThreads), kVertThreads, s);
}

// Eager substep with the convergence test (profiling): the host reads the
// decision of k_check_converged after every chunk.
int run_step_tol_eager(AdmmB200* h, float tol) {
    DevScene& s = h->s;
    enqueue_step_begin(h);
    cudaMemsetAsync(s.done, 0, sizeof(int) * 4, h->cstream);
    const int k = h->chunk;
    for (int c = 0;; c++) {
        for (int it = 0; it < k; it++) enqueue_iteration(h, it, c == 0 && it == 0, it == k - 1);
        LAUNCH(k_check_converged, 1, 32, s, cudaGraphConditionalHandle(0), tol, k, h->admm_max_iter, 0);
        int more = 0;
        CK(cudaMemcpyAsync(&more, s.done + 1, sizeof(int), cudaMemcpyDeviceToHost, h->cstream));
        CK(cudaStreamSynchronize(h->cstream));
        if (!more) break;
    }
    enqueue_step_end(h);
    return ADMM_OK;
}

// Substep with a convergence test (residual_tol > 0): the first chunk of
// h->chunk iterations, then a WHILE node of the graph whose body runs further
// chunks while k_check_converged keeps its condition set.
int enqueue_step_tol(AdmmB200* h, float tol) {
    DevScene& s = h->s;
    enqueue_step_begin(h);
    cudaMemsetAsync(s.done, 0, sizeof(int) * 4, h->cstream);
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    CK(cudaStreamGetCaptureInfo(h->cstream, &cst, nullptr, &g, nullptr, nullptr));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    const int k = h->chunk;
    for (int it = 0; it < k; it++) enqueue_iteration(h, it, it == 0, it == k - 1);
    LAUNCH(k_check_converged, 1, 32, s, cond, tol, k, h->admm_max_iter, 1);
    // WHILE node after everything captured so far
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(h->cstream, &cst, nullptr, &g, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    CK(cudaGraphAddNode(&wnode, g, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    // the body: one more chunk, captured from a second stream into the body graph
    cudaStream_t parent = h->cstream;
    h->cstream = h->body_stream;
    h->in_body = true;
    const int before = h->launch_counter;
    CK(cudaStreamBeginCaptureToGraph(h->cstream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < k; it++) enqueue_iteration(h, it, false, it == k - 1);
    LAUNCH(k_check_converged, 1, 32, s, cond, tol, k, h->admm_max_iter, 1);
    h->kernels_body = h->launch_counter - before;
    h->launch_counter = before;
    h->in_body = false;
    cudaGraph_t bg = nullptr;
    CK(cudaStreamEndCapture(h->cstream, &bg));
    h->cstream = parent;
    CK(cudaStreamUpdateCaptureDependencies(h->cstream, &wnode, 1, cudaStreamSetCaptureDependencies));
    enqueue_step_end(h);
    return ADMM_OK;
}

// One substep (ADMMImplGPU::step).  The residual of the last iteration is kept.
void enqueue_step(AdmmB200* h) {
    DevScene& s = h->s;
    enqueue_step_begin(h);
    for (int it = 0; it < h->admm_max_iter; it++) enqueue_iteration(h, it, it == 0, it == h->admm_max_iter - 1);
    if (h->admm_max_iter > 0) enqueue_local(h, LOCAL_DUAL);
    set_phase(h, ADMM_PHASE_FINAL);
    LAUNCH(k_vertex_final, blocks(s.n, kVertThreads), kVertThreads, s);
}

int build_step_graph_once(AdmmB200* h) {
    if (h->probe_kernel == ADMM_PROBE_PHASES && h->pev.empty()) {
        h->pev.resize(kMaxPhaseEvents);
        h->pev_phase.resize(kMaxPhaseEvents);
        h->pev_launch.resize(kMaxPhaseEvents);
        for (auto& e : h->pev) CK(cudaEventCreate(&e));
    } else if (h->probe_kernel != 0 && h->probe_kernel != ADMM_PROBE_PHASES && h->probe_ev.empty()) {
        h->probe_ev.resize(2 * kMaxProbes);
        for (auto& e : h->probe_ev) CK(cudaEventCreate(&e));
    }
    h->probe_used = 0;
    h->pev_used = 0;
    h->phase = -1;
    cudaGraph_t g = nullptr;
    h->cstream = h->stream;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->launch_counter = 0;
    h->enqueue_rc = ADMM_OK;
    int rc = ADMM_OK;
    if (h->residual_tol > 0.f) rc = enqueue_step_tol(h, h->residual_tol);
    else enqueue_step(h);
    if (rc == ADMM_OK) rc = h->enqueue_rc;
    set_phase(h, ADMM_NUM_PHASES);  // closes the last phase
    h->kernels_per_step = h->launch_counter;
    cudaError_t ee = cudaStreamEndCapture(h->stream, &g);
    if (rc != ADMM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    CK(ee);
    cudaError_t e = cudaGraphInstantiate(&h->step_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->step_exec = nullptr;
        return fail(h, ADMM_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    return ADMM_OK;
}

// Captures and instantiates the substep graph.  Should the runtime refuse the
// cooperative persistent kernel inside a graph (or inside a conditional body),
// the graph is built again with one kernel per sweep.
int build_step_graph(AdmmB200* h) {
    if (h->step_exec) return ADMM_OK;
    const int rc = build_step_graph_once(h);
    if (rc == ADMM_OK || !h->persist) return rc;
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    for (cudaStream_t st : {h->if_stream, h->body_stream, h->stream})
        if (cudaStreamIsCapturing(st, &cst) == cudaSuccess && cst != cudaStreamCaptureStatusNone) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            g = nullptr;
        }
    cudaGetLastError();
    h->cstream = h->stream;
    h->in_body = false;
    fprintf(stderr, "admm_b200: persistent global step not capturable (%s); using one kernel per sweep\n",
            h->last_error.c_str());
    h->persist = false;
    return build_step_graph_once(h);
}

bool learned_active(const AdmmB200* h) { return h->global_solver == 3; }

// One substep from its graph (a learned substep judges and replaces its failed
// solves inside the graph).
int launch_substep(AdmmB200* h) {
    CK(cudaGraphLaunch(h->step_exec, h->stream));
    if (learned_active(h)) h->learn_substeps++;
    return ADMM_OK;
}

// The eager (profiling / recording) substep.
int run_substep_eager(AdmmB200* h) {
    h->cstream = h->stream;
    if (h->residual_tol > 0.f) TRY(run_step_tol_eager(h, h->residual_tol));
    else enqueue_step(h);
    CK(cudaGetLastError());
    TRY(h->enqueue_rc);
    if (learned_active(h)) h->learn_substeps++;
    return ADMM_OK;
}

float4 pack(const float* p) { return make_float4(p[0], p[1], p[2], 0.f); }

// The caller's index of internal vertex i (identity without renumbering).
inline int caller_of(const AdmmB200* h, int i) { return h->perm.empty() ? i : h->perm[i]; }

// Buffers with one row per vertex (the others have one per constraint row).
inline bool per_vertex_buffer(int which) {
    return which == ADMM_BUF_X || which == ADMM_BUF_X0 || which == ADMM_BUF_V || which == ADMM_BUF_P ||
           which == ADMM_BUF_UC || which == ADMM_BUF_B || which == ADMM_BUF_MXT;
}

float4* buffer_ptr(AdmmB200* h, int which, int* rows) {
    DevScene& s = h->s;
    switch (which) {
        case ADMM_BUF_X: *rows = s.n; return s.x;
        case ADMM_BUF_X0: *rows = s.n; return s.x0;
        case ADMM_BUF_V: *rows = s.n; return s.v;
        case ADMM_BUF_P: *rows = s.n; return s.p;
        case ADMM_BUF_UC: *rows = s.nd; return s.uc;
        case ADMM_BUF_UE: *rows = s.m; return s.ue;
        case ADMM_BUF_Z: *rows = s.m; return s.z;
        case ADMM_BUF_B: *rows = s.nd; return s.b;
        case ADMM_BUF_MXT: *rows = s.n; return s.mxt;
    }
    *rows = 0;
    return nullptr;
}

int upload_state(AdmmB200* h, const std::vector<float4>& x, const std::vector<float4>& v) {
    DevScene& s = h->s;
    CK(cudaMemcpyAsync(s.x0, x.data(), sizeof(float4) * s.n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(s.x, x.data(), sizeof(float4) * s.n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(s.v, v.data(), sizeof(float4) * s.n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

// Grid parameters from the rest shape: cell edge = max(2.05 x thickness, 1.5 x
// the median of the surface elements' largest box extent), so that a vertex
// query spans at most 2 cells per axis and most elements 1-2, while a few large
// elements (a ground plane, a collider box) go to the big lists; buckets = twice
// the rest insertions (power of two); entry capacity = 4x them (elements
// beyond it fall back to the big lists).
int setup_grid(AdmmB200* h, const AdmmB200Desc* d) {
    DevScene& s = h->s;
    GridDev& g = s.grid;
    const int ne = s.nst + s.nse;
    std::vector<float> ext;
    std::vector<float4> lo(ne), up(ne);
    ext.reserve(ne);
    auto box = [&](int u, const int* v, int nv) {
        float4 a = make_float4(1e32f, 1e32f, 1e32f, 0.f), b = make_float4(-1e32f, -1e32f, -1e32f, 0.f);
        for (int k = 0; k < nv; k++) {
            const float4 p = h->x_init[v[k]];
            a.x = std::min(a.x, p.x); a.y = std::min(a.y, p.y); a.z = std::min(a.z, p.z);
            b.x = std::max(b.x, p.x); b.y = std::max(b.y, p.y); b.z = std::max(b.z, p.z);
        }
        lo[u] = a;
        up[u] = b;
        ext.push_back(std::max(b.x - a.x, std::max(b.y - a.y, b.z - a.z)));
    };
    for (int f = 0; f < s.nst; f++) box(f, d->surf_tris + 3 * f, 3);
    for (int e = 0; e < s.nse; e++) box(s.nst + e, d->surf_edges + 2 * e, 2);
    float c = 2.05f * s.thickness;
    if (!ext.empty()) {
        const size_t k = (ext.size() - 1) / 2;
        std::nth_element(ext.begin(), ext.begin() + k, ext.end());
        c = std::max(c, 1.5f * ext[k]);
    }
    if (!(c > 0.f) || !std::isfinite(c)) c = 1.f;
    g.inv_c = 1.f / c;
    h->grid_cell_size = c;
    int64_t ins = 0;
    for (int u = 0; u < ne; u++) {
        int64_t cells = 1;
        const float a[3] = {lo[u].x, lo[u].y, lo[u].z}, b[3] = {up[u].x, up[u].y, up[u].z};
        for (int k = 0; k < 3; k++) {
            const int64_t span = (int64_t)std::floor(b[k] * g.inv_c) - (int64_t)std::floor(a[k] * g.inv_c) + 1;
            cells = span <= kGridMaxSpan ? cells * span : 0;
        }
        ins += cells;
    }
    int64_t nb = 1024;
    while (nb < 2 * ins) nb <<= 1;
    if (nb > (int64_t(1) << 28)) return fail(h, ADMM_ERR_INVALID, "collision grid too large");
    g.hmask = (int)nb - 1;
    h->grid_buckets = (int)nb;
    g.cap = (int)std::min<int64_t>(4 * ins + 4096, int64_t(1) << 30);
    TRY(dalloc(h, &g.cnt, nb));
    TRY(dalloc(h, &g.start, nb + 1));
    TRY(dalloc(h, &g.ent_lo, g.cap));
    TRY(dalloc(h, &g.ent_up, g.cap));
    TRY(dalloc(h, &g.ent_key, g.cap));
    TRY(dalloc(h, &g.ctr, 4));
    TRY(dalloc(h, &g.big_tri, std::max(s.nst, 1)));
    TRY(dalloc(h, &g.big_edge, std::max(s.nse, 1)));
    TRY(dalloc(h, &g.mode, std::max(ne, 1)));
    TRY(dalloc(h, &g.qkey, std::max(s.cap, 1)));
    TRY(dalloc(h, &g.qhits, (size_t)std::max(s.nsv + s.nse, 1) * kQueryHitsMax));
    // lanes per query: 32 while 32 lanes per query fill at most four waves of
    // the device, else 16 or 8 (a detection of millions of queries is bound by
    // throughput, not by the latency of one query's loads)
    if (d->query_lanes != 0) {
        h->query_lanes = d->query_lanes;
    } else {
        int sms = 148;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
        const int64_t four_waves = 4ll * sms * 2048;
        const int64_t nq = s.nsv + s.nse;
        h->query_lanes = nq * 32 <= four_waves ? 32 : nq * 16 <= four_waves ? 16 : 8;
    }
    return ADMM_OK;
}

int create_impl(const AdmmB200Desc* d, int device, AdmmB200* h) {
    if (d->abi_version != ADMM_B200_ABI_VERSION) return fail(h, ADMM_ERR_INVALID, "abi_version");
    if (!d->x0 || !d->mass) return fail(h, ADMM_ERR_INVALID, "x0/mass");
    if (d->enable_contact && !d->contact_w) return fail(h, ADMM_ERR_INVALID, "contact_w");
    if (d->n_tri && (!d->tri_inds || !d->tri_binv || !d->tri_w)) return fail(h, ADMM_ERR_INVALID, "tri arrays");
    if (d->n_tet && (!d->tet_inds || !d->tet_binv || !d->tet_w)) return fail(h, ADMM_ERR_INVALID, "tet arrays");
    if (d->n_bend && (!d->bend_offsets || !d->bend_inds || !d->bend_coeffs || !d->bend_w))
        return fail(h, ADMM_ERR_INVALID, "bend arrays");
    if (d->n_pin && (!d->pin_inds || !d->pin_pos || !d->pin_w)) return fail(h, ADMM_ERR_INVALID, "pin arrays");
    if (!(d->dt > 0.f)) return fail(h, ADMM_ERR_INVALID, "dt");
    if (d->admm_max_iter < 0 || d->gs_max_iter < 0 || d->jacobi_iter < 0) return fail(h, ADMM_ERR_INVALID, "iteration counts");
    if (d->enable_contact && d->max_contacts <= 0) return fail(h, ADMM_ERR_INVALID, "max_contacts");
    if (d->query_lanes != 0 && d->query_lanes != 8 && d->query_lanes != 16 && d->query_lanes != 32)
        return fail(h, ADMM_ERR_INVALID, "query_lanes");
    if (d->contact_semantics != 0 && d->contact_semantics != 1) return fail(h, ADMM_ERR_INVALID, "contact_semantics");
    if (d->backend_semantics != 0 && d->backend_semantics != 1) return fail(h, ADMM_ERR_INVALID, "backend_semantics");
    if (d->backend_semantics == 1 && !(d->damp_k_L >= 0.f && d->damp_k_M >= 0.f))
        return fail(h, ADMM_ERR_INVALID, "damp_k_L/damp_k_M");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return fail(h, ADMM_ERR_NO_DEVICE, "no CUDA device");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(h, ADMM_ERR_NO_DEVICE, "device is not sm_100 (Blackwell B200)");
    CK(cudaSetDevice(device));
    h->device = device;
    // ADMM_B200_PDL=0 launches every kernel of a substep without programmatic dependent
    // launch (each kernel then starts after its predecessor completes); results are
    // the same bits either way, which the tests check.
    if (const char* e = std::getenv("ADMM_B200_PDL")) h->pdl = !(e[0] == '0' && e[1] == '\0');

    Assembly as;
    std::string why = assemble(*d, as);
    if (!why.empty()) return fail(h, ADMM_ERR_INVALID, why);

    DevScene& s = h->s;
    s.n = d->n_vert; s.nd = d->n_dyn; s.m = d->n_rows;
    s.ntri = d->n_tri; s.ntet = d->n_tet; s.nbend = d->n_bend; s.npin = d->n_pin;
    s.tri_sr = d->tri_start_row; s.tet_sr = d->tet_start_row; s.bend_sr = d->bend_start_row; s.pin_sr = d->pin_start_row;
    s.dt = d->dt;
    s.dt_inv = 1.0f / d->dt;
    s.g = d->g;
    s.mu = d->mu;
    s.eps = 1.0f / (d->dt * d->dt * d->kappa + d->dt * d->beta);   // admm_impl_gpu.cu:259
    s.gam = d->dt * d->kappa / (d->dt * d->kappa + d->beta);        // admm_impl_gpu.cu:260
    s.thickness = d->thickness;
    s.contact = d->enable_contact ? 1 : 0;
    h->admm_max_iter = d->admm_max_iter;
    h->dcd_interval = d->dcd_interval > 0 ? d->dcd_interval : 1;
    h->gs_iter = d->gs_max_iter;
    h->jac_iter = d->jacobi_iter;
    h->residual_tol = d->residual_tol;
    h->warmstart_ue = d->warmstart_ue != 0;
    h->bvh_refit = d->bvh_refit != 0;
    h->warmstart_uc = d->warmstart_uc != 0;
    h->residual_every = d->residual_check_every;
    const int n = s.n, nd = s.nd, m = s.m;

    // vertex state
    h->x_init.resize(n);
    h->v_init.assign(n, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int i = 0; i < n; i++) {
        h->x_init[i] = pack(d->x0 + 3 * i);
        if (d->v0) h->v_init[i] = pack(d->v0 + 3 * i);
    }
    TRY(dalloc(h, &s.x, n));
    TRY(dalloc(h, &s.x0, n));
    TRY(dalloc(h, &s.v, n));
    TRY(dalloc(h, &s.p, n));
    TRY(dalloc(h, &s.mxt, n));
    TRY(dalloc(h, &s.b, nd));
    TRY(dalloc(h, &s.uc, nd));
    TRY(dalloc(h, &s.xprev, n));
    TRY(dalloc(h, &s.jac[0], nd));
    TRY(dalloc(h, &s.jac[1], nd));
    float* mass = nullptr;
    int* fixed = nullptr;
    TRY(dupload(h, &mass, d->mass, n));
    std::vector<int> fx(n, 0);
    if (d->is_fixed) for (int i = 0; i < n; i++) fx[i] = d->is_fixed[i];
    TRY(dupload(h, &fixed, fx.data(), n));
    s.mass = mass;
    s.fixed = fixed;
    float *dt2wc = nullptr, *cw = nullptr, *cwinv = nullptr;
    TRY(dupload(h, &dt2wc, as.dt2wc.data(), nd));
    std::vector<float> hcw(n, 1e12f), hcwi(n, 0.f);
    if (d->contact_w)
        for (int i = 0; i < n; i++) {
            hcw[i] = d->contact_w[i];
            hcwi[i] = i < nd ? 1.0f / hcw[i] : 0.f;  // solver_config_applier.cpp:36-46
        }
    TRY(dupload(h, &cw, hcw.data(), n));
    TRY(dupload(h, &cwinv, hcwi.data(), n));
    s.dt2wc = dt2wc; s.cw = cw; s.cwinv = cwinv;

    // constraints
    {
        std::vector<int4> ti(s.ntri);
        std::vector<float4> tb(s.ntri);
        for (int c = 0; c < s.ntri; c++) {
            ti[c] = make_int4(d->tri_inds[3 * c], d->tri_inds[3 * c + 1], d->tri_inds[3 * c + 2], 0);
            const float* B = d->tri_binv + 4 * c;
            tb[c] = make_float4(B[0], B[1], B[2], B[3]);
        }
        int4* a; float4* b;
        TRY(dupload(h, &a, ti.data(), s.ntri)); TRY(dupload(h, &b, tb.data(), s.ntri));
        s.tri_inds = a; s.tri_binv = b;
    }
    {
        std::vector<int4> ti(s.ntet);
        std::vector<float4> b0(s.ntet), b1(s.ntet), b2(s.ntet);
        for (int c = 0; c < s.ntet; c++) {
            const int* id = d->tet_inds + 4 * c;
            ti[c] = make_int4(id[0], id[1], id[2], id[3]);
            const float* B = d->tet_binv + 9 * c;
            b0[c] = make_float4(B[0], B[1], B[2], 0.f);
            b1[c] = make_float4(B[3], B[4], B[5], 0.f);
            b2[c] = make_float4(B[6], B[7], B[8], 0.f);
        }
        int4* a; float4 *p0, *p1, *p2;
        TRY(dupload(h, &a, ti.data(), s.ntet));
        TRY(dupload(h, &p0, b0.data(), s.ntet)); TRY(dupload(h, &p1, b1.data(), s.ntet)); TRY(dupload(h, &p2, b2.data(), s.ntet));
        s.tet_inds = a; s.tet_b0 = p0; s.tet_b1 = p1; s.tet_b2 = p2;
    }
    {
        const int ne = s.nbend ? d->bend_offsets[s.nbend] : 0;
        int *o, *ii; float *cf, *rn;
        std::vector<int> off(s.nbend + 1, 0);
        if (s.nbend) std::memcpy(off.data(), d->bend_offsets, sizeof(int) * (s.nbend + 1));
        TRY(dupload(h, &o, off.data(), s.nbend + 1));
        TRY(dupload(h, &ii, d->bend_inds, ne));
        TRY(dupload(h, &cf, d->bend_coeffs, ne));
        std::vector<float> rest(s.nbend, 0.f);
        if (d->bend_rest_norm) for (int c = 0; c < s.nbend; c++) rest[c] = d->bend_rest_norm[c];
        TRY(dupload(h, &rn, rest.data(), s.nbend));
        s.bend_off = o; s.bend_inds = ii; s.bend_coef = cf; s.bend_rest = rn;
    }
    {
        int* pi; float4* pp;
        std::vector<float4> pos(s.npin);
        for (int c = 0; c < s.npin; c++) pos[c] = pack(d->pin_pos + 3 * c);
        TRY(dupload(h, &pi, d->pin_inds, s.npin));
        TRY(dupload(h, &pp, pos.data(), s.npin));
        s.pin_inds = pi; s.pin_pos = pp;
    }
    float* wrow;
    TRY(dupload(h, &wrow, as.wrow.data(), m));
    s.wrow = wrow;
    TRY(dalloc(h, &s.z, m));
    TRY(dalloc(h, &s.ue, m));
    TRY(dalloc(h, &s.y, m));
    // matrices (sliced-ELL layouts are chosen by the autotuner below)
    {
        float* dg;
        TRY(dupload(h, &dg, as.a_diag.data(), nd));
        s.a_diag = dg;
    }
    // collision geometry and contacts
    s.nst = d->enable_contact ? d->n_surf_tri : 0;
    s.nse = d->enable_contact ? d->n_surf_edge : 0;
    s.nsv = d->enable_contact ? d->n_surf_vert : 0;
    {
        std::vector<int4> st(s.nst);
        for (int f = 0; f < s.nst; f++) {
            const int* t = d->surf_tris + 3 * f;
            for (int k = 0; k < 3; k++)
                if (t[k] < 0 || t[k] >= n) return fail(h, ADMM_ERR_INVALID, "surf_tris out of range");
            st[f] = make_int4(t[0], t[1], t[2], 0);
        }
        std::vector<int2> se(s.nse);
        for (int e = 0; e < s.nse; e++) {
            const int* t = d->surf_edges + 2 * e;
            if (t[0] < 0 || t[0] >= n || t[1] < 0 || t[1] >= n) return fail(h, ADMM_ERR_INVALID, "surf_edges out of range");
            se[e] = make_int2(t[0], t[1]);
        }
        int4* a; int2* b; int* c;
        TRY(dupload(h, &a, st.data(), s.nst));
        TRY(dupload(h, &b, se.data(), s.nse));
        TRY(dupload(h, &c, d->surf_verts, s.nsv));
        s.st = a; s.se = b; s.sv = c;
    }
    s.cap = d->enable_contact ? d->max_contacts : 1;
    TRY(dalloc(h, &s.nc, 1));
    TRY(dalloc(h, &s.nc_raw, 1));
    TRY(dalloc(h, &s.err, 4));
    TRY(dalloc(h, &s.pairs, s.cap));
    TRY(dalloc(h, &s.bary, s.cap));
    TRY(dalloc(h, &s.nrm, s.cap));
    TRY(dalloc(h, &s.point, s.cap));
    TRY(dalloc(h, &s.gamma, s.cap));
    TRY(dalloc(h, &s.kc, s.cap));
    TRY(dalloc(h, &s.rc, s.cap));
    TRY(dalloc(h, &s.cmu, s.cap));
    if (d->vert_mu) {
        for (int i = 0; i < n; i++)
            if (!(d->vert_mu[i] >= 0.f)) return fail(h, ADMM_ERR_INVALID, "vert_mu must be >= 0");
        float* vm;
        TRY(dupload(h, &vm, d->vert_mu, n));
        s.vmu = vm;
    }
    TRY(dalloc(h, &s.ginc, 4 * (size_t)s.cap));
    TRY(dalloc(h, &s.cinc, 4 * (size_t)s.cap));
    TRY(dalloc(h, &s.vtmp, 4 * (size_t)s.cap));
    TRY(dalloc(h, &s.du, s.cap));
    TRY(dalloc(h, &s.du2, s.cap));
    TRY(dalloc(h, &s.p2, n));
    TRY(dalloc(h, &s.vcnt, n));
    TRY(dalloc(h, &s.vfill, n));
    TRY(dalloc(h, &s.vstart, n + 1));
    TRY(dalloc(h, &s.vlist, 4 * (size_t)s.cap));
    TRY(alloc_bvh(h, s.bf, s.nst));
    TRY(alloc_bvh(h, s.be, s.nse));
    TRY(dalloc(h, &s.qcount, s.nsv + s.nse + 1));
    TRY(dalloc(h, &s.qoff, s.nsv + s.nse + 1));
    h->sort_max = std::max(s.nst, s.nse);
    const int hist_n = 256 * sort_tiles(std::max(h->sort_max, 1));
    TRY(dalloc(h, &h->hist, hist_n));
    if (d->broad_phase < 0 || d->broad_phase > 2) return fail(h, ADMM_ERR_INVALID, "broad_phase must be 0, 1 or 2");
    s.cpu_backend = d->backend_semantics == 1 ? 1 : 0;
    s.cpu_contact = (d->contact_semantics == 1 || s.cpu_backend) ? 1 : 0;
    h->use_grid = d->broad_phase != 1 || s.cpu_contact;  // the CPU predicates run on the grid
    if (s.cpu_backend) {
        int* ds = nullptr;
        int* dc = nullptr;
        float* dv = nullptr;
        float* dd = nullptr;
        std::vector<float> vals(as.damp.val.begin(), as.damp.val.end());
        TRY(dupload(h, &ds, as.damp.start.data(), as.damp.start.size()));
        TRY(dupload(h, &dc, as.damp.col.empty() ? nullptr : as.damp.col.data(), std::max<size_t>(as.damp.col.size(), 1)));
        TRY(dupload(h, &dv, vals.empty() ? nullptr : vals.data(), std::max<size_t>(vals.size(), 1)));
        TRY(dupload(h, &dd, as.damp_diag.data(), as.damp_diag.size()));
        s.dmp_start = ds;
        s.dmp_col = dc;
        s.dmp_val = dv;
        s.dmp_diag = dd;
    }

    TRY(setup_grid(h, d));
    const int scan_n = std::max(std::max(std::max(scan_tiles(hist_n), scan_tiles(n + 1)), scan_tiles(s.nsv + s.nse + 1)),
                                scan_tiles(h->grid_buckets)) + 4;
    TRY(dalloc(h, &s.scan_tmp, scan_n));
    TRY(dalloc(h, &s.res, 4));
    TRY(dalloc(h, &s.done, 4));
    h->contact_grid = std::max(1, std::min(blocks(s.cap, kContactThreads), 2 * 148));
    h->group_grid = std::max(1, std::min(blocks(std::min(n, 4 * s.cap) * kGatherLanes, kContactThreads), 8 * 148));
    // one wave of three blocks per SM (the pass holds 74 registers per thread): a warp per contact
    // over a grid-stride loop; with a few hundred contacts most blocks only start and exit, and
    // 8 * 148 of them cost a quarter more per launch than 4 * 148
    h->pass_grid = std::max(1, std::min(blocks(s.cap * 32, kContactThreads), 3 * 148));
    h->warp_grid = std::max(1, std::min(blocks(std::min(n, 4 * s.cap) * 32, kContactThreads), 8 * 148));
    TRY(dalloc(h, &s.tpos, n));
    TRY(dalloc(h, &s.tv, n));
    TRY(dalloc(h, &s.tvr, n));
    TRY(dalloc(h, &s.ntv, 1));

    h->tet_blocks = s.ntet ? blocks(s.ntet, kLocalThreads) : 0;
    h->tri_blocks = s.ntri ? blocks(s.ntri, kLocalThreads) : 0;
    h->bend_blocks = s.nbend ? blocks(s.nbend, kLocalThreads) : 0;
    h->pin_blocks = s.npin ? blocks(s.npin, kLocalThreads) : 0;
    if (h->tet_blocks + h->tri_blocks + h->bend_blocks + h->pin_blocks == 0) return fail(h, ADMM_ERR_INVALID, "no constraints");
    TRY(dalloc(h, &s.res_part, 3 * (size_t)(h->tet_blocks + h->tri_blocks + h->bend_blocks + h->pin_blocks +
                                            blocks(s.nd, kLocalThreads))));

    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->body_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->if_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));

    h->cstream = h->stream;
    {
        const int every = d->residual_check_every > 0 ? d->residual_check_every : h->dcd_interval;
        h->chunk = (every + h->dcd_interval - 1) / h->dcd_interval * h->dcd_interval;
        if (h->residual_tol > 0.f && h->chunk > h->admm_max_iter)
            return fail(h, ADMM_ERR_INVALID, "residual_check_every/dcd_interval exceed admm_max_iter");
    }
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    TRY(upload_state(h, h->x_init, h->v_init));
    if (d->ell_lanes != 0 && d->ell_lanes != 1 && d->ell_lanes != 2 && d->ell_lanes != 4 && d->ell_lanes != 8)
        return fail(h, ADMM_ERR_INVALID, "ell_lanes must be 0, 1, 2, 4 or 8");
    TRY(autotune_ell(h, as, d->ell_lanes, &h->tune_lanes_a, &h->tune_lanes_r, &h->tune_ms_a, &h->tune_ms_r));
    if (d->jacobi_mode < 0 || d->jacobi_mode > 3) return fail(h, ADMM_ERR_INVALID, "jacobi_mode must be 0, 1, 2 or 3");
    if (d->global_solver < 0 || d->global_solver > 3) return fail(h, ADMM_ERR_INVALID, "global_solver must be 0, 1, 2 or 3");
    if (d->pcg_iter < 0) return fail(h, ADMM_ERR_INVALID, "pcg_iter");
    h->global_solver = d->global_solver;
    h->pcg_iter = d->pcg_iter > 0 ? d->pcg_iter : std::max(1, d->jacobi_iter / 2);
    {
        PcgDev& g = h->pcg;
        TRY(dalloc(h, &g.r, nd));
        TRY(dalloc(h, &g.u, nd));
        TRY(dalloc(h, &g.w, nd));
        TRY(dalloc(h, &g.p, nd));
        TRY(dalloc(h, &g.s, nd));
        g.blocks = blocks(s.A.nslices * 32, kVertThreads);
        TRY(dalloc(h, &g.part, 2 * (size_t)g.blocks));
        TRY(dalloc(h, &g.scal, 8));
    }
    {
        // learned global step: the Jacobi sweep until admm_b200_set_learned (m = 1 / a_ii)
        LearnDev& L = h->learn;
        L.blocks = blocks(s.A.nslices * 32, kVertThreads);
        float* minv = nullptr;
        float* theta = nullptr;
        TRY(dalloc(h, &minv, nd));
        TRY(dalloc(h, &theta, nd));
        std::vector<float> mv(nd);
        for (int i = 0; i < nd; i++) mv[i] = 1.f / as.a_diag[i];
        CK(cudaMemcpy(minv, mv.data(), sizeof(float) * nd, cudaMemcpyHostToDevice));
        L.minv = minv;
        L.theta = theta;
        TRY(dalloc(h, &L.xl, nd));
        L.rblocks = blocks(s.R.nslices * 32, kVertThreads);
        TRY(dalloc(h, &L.ax, nd));
        TRY(dalloc(h, &L.part, 3 * (size_t)L.blocks));
        TRY(dalloc(h, &L.part_c, (size_t)L.blocks));
        TRY(dalloc(h, &L.stats, 4));
        TRY(dalloc(h, &L.fail, 1));
        TRY(dalloc(h, &L.warm, 1));
        CK(cudaHostAlloc((void**)&h->fail_host, sizeof(int), cudaHostAllocDefault));
        h->learn_sweeps = std::max(1, h->jac_iter);
        h->learn_omega.assign(h->learn_sweeps, 1.f);
        h->learn_beta.assign(h->learn_sweeps, 0.f);
    }
    h->hostA = as.A;
    h->hostAdiag = as.a_diag;
    TRY(build_persist_plan(h, as.A));
    TRY(build_tiles_dev(h, as.A));
    h->persist = h->tiled = false;
    if (h->jac_iter >= 2 && (d->global_solver == 0 || d->global_solver == 3)) {
        if (d->jacobi_mode == 2 && h->persist_ok) {
            h->persist = true;
        } else if (d->jacobi_mode == 3) {
            h->tiled = true;
        } else if (d->jacobi_mode == 0) {
            TRY(time_global(h, 1, &h->tune_ms_sweeps));
            TRY(time_global(h, 3, &h->tune_ms_tiled));
            if (h->persist_ok) TRY(time_global(h, 2, &h->tune_ms_persist));
            float best = h->tune_ms_sweeps;
            if (h->tune_ms_tiled < best) {
                best = h->tune_ms_tiled;
                h->tiled = true;
            }
            if (h->persist_ok && h->tune_ms_persist < best) {
                h->tiled = false;
                h->persist = true;
            }
        }
    }
    TRY(upload_state(h, h->x_init, h->v_init));
    return ADMM_OK;
}

// Host-order staging buffer (row-major n x 3 positions, then velocities) <-> the
// internal float4 state; perm[i] = the caller's row of internal vertex i (null: identity).
__global__ void k_unpack_state(DevScene s, const float* __restrict__ stage, int has_v, const int* __restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    const int c = perm ? perm[i] : i;
    const float4 x = make_float4(stage[3 * c], stage[3 * c + 1], stage[3 * c + 2], 0.f);
    s.x0[i] = x;
    s.x[i] = x;
    if (has_v) s.v[i] = make_float4(stage[3 * s.n + 3 * c], stage[3 * s.n + 3 * c + 1], stage[3 * s.n + 3 * c + 2], 0.f);
}

__global__ void k_pack_state(DevScene s, float* __restrict__ stage, const int* __restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    const int c = perm ? perm[i] : i;
    const float4 x = s.x0[i], v = s.v[i];
    stage[3 * c] = x.x; stage[3 * c + 1] = x.y; stage[3 * c + 2] = x.z;
    stage[3 * s.n + 3 * c] = v.x; stage[3 * s.n + 3 * c + 1] = v.y; stage[3 * s.n + 3 * c + 2] = v.z;
}

int accumulate_timers(AdmmB200* h) {
    if (h->profiling) {
        for (int k = 0; k + 1 < h->prof_used; k += 2) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->prof_ev[k], h->prof_ev[k + 1]));
            const int ph = h->prof_phase[k / 2];
            if (ph < 0 || ph >= ADMM_NUM_PHASES) continue;
            h->phase_ms[ph] += ms;
            h->phase_launches[ph] += 1;
        }
        h->prof_used = 0;
    } else if (h->probe_kernel == ADMM_PROBE_PHASES) {
        for (int k = 0; k + 1 < h->pev_used; k++) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->pev[k], h->pev[k + 1]));
            const int ph = h->pev_phase[k];
            if (ph < 0 || ph >= ADMM_NUM_PHASES) continue;
            h->phase_ms[ph] += ms;
            h->phase_launches[ph] += h->pev_launch[k + 1] - h->pev_launch[k];
        }
    } else if (h->probe_kernel != 0) {
        for (int k = 0; k + 1 < h->probe_used; k += 2) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->probe_ev[k], h->probe_ev[k + 1]));
            h->probe_ms += ms;
            h->probe_n += 1;
        }
    }
    return ADMM_OK;
}

int read_err_flags(AdmmB200* h, int* status) {
    int e[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(e, h->s.err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e[0] || e[1] || e[2] || e[3]) CK(cudaMemset(h->s.err, 0, sizeof(int) * 4));
    // after a timed-out wait the blocks' sweep counters disagree: start them again from 0
    if (e[3] && h->pp.epoch) CK(cudaMemset(h->pp.epoch, 0, sizeof(unsigned) * h->pp.blocks));
    *status = e[3] ? ADMM_ERR_TIMEOUT : e[0] ? ADMM_ERR_CONTACT_OVERFLOW : e[1] ? ADMM_ERR_STACK_OVERFLOW
            : e[2] ? ADMM_ERR_NAN : ADMM_OK;
    return ADMM_OK;
}

}  // namespace

// ================================ C ABI =====================================
// Scripted static meshes: publish the track records to the device, place the
// meshes at their first frame (the animate_all of ADMMImplGPU::init / reset)
// and drop the step graph, which holds the track count.
int anim_publish(AdmmB200* h) {
    AnimDev& a = h->anim;
    if (!a.tracks) {
        TRY(dalloc(h, &a.tracks, kMaxTracks));
        TRY(dalloc(h, &a.counter, 1));
        TRY(dalloc(h, &a.frame, kMaxTracks));
        TRY(dalloc(h, &a.moving, kMaxTracks));
    }
    int first = 0;
    for (auto& t : h->tracks) {
        t.first = first;
        first += t.v1 - t.v0;
    }
    a.n_tracks = (int)h->tracks.size();
    a.n_verts = first;
    if (a.n_tracks)
        CK(cudaMemcpy(a.tracks, h->tracks.data(), sizeof(TrackDev) * h->tracks.size(), cudaMemcpyHostToDevice));
    if (h->step_exec) {
        cudaGraphExecDestroy(h->step_exec);
        h->step_exec = nullptr;
    }
    return ADMM_OK;
}

int anim_init(AdmmB200* h) {
    if (h->anim.n_tracks == 0) return ADMM_OK;
    h->cstream = h->stream;
    LAUNCH(k_anim_advance, 1, 32, h->anim, 1);
    LAUNCH(k_animate, blocks(h->anim.n_verts, kVertThreads), kVertThreads, h->s, h->anim);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

int add_track(AdmmB200* h, TrackDev t) {
    if ((int)h->tracks.size() >= kMaxTracks) return fail(h, ADMM_ERR_INVALID, "too many tracks");
    for (const auto& o : h->tracks)
        if (t.v0 < o.v1 && o.v0 < t.v1) return fail(h, ADMM_ERR_INVALID, "track vertex ranges overlap");
    h->tracks.push_back(t);
    TRY(anim_publish(h));
    return anim_init(h);
}

int check_track_range(AdmmB200* h, int v0, int v1, int n_frames) {
    if (v0 < h->s.nd || v1 > h->s.n || v0 >= v1) return fail(h, ADMM_ERR_INVALID, "track range must be static vertices");
    if (n_frames < 1) return fail(h, ADMM_ERR_INVALID, "n_frames");
    return ADMM_OK;
}

// The renumbered copy of a description (arrays owned here, pointers in d).
struct RenumberedDesc {
    AdmmB200Desc d;
    std::vector<float> x0, v0, mass, cw, vmu;
    std::vector<int32_t> fixed, tri, tet, bend, pin, st, se, sv;
};

// Every vertex index of the description in range (else no renumbering: create reports it).
bool indices_in_range(const AdmmB200Desc* d) {
    const int n = d->n_vert, nd = d->n_dyn;
    if (n <= 0 || nd <= 0 || nd > n) return false;
    auto ok = [](const int32_t* a, size_t cnt, int hi) {
        if (cnt && !a) return false;
        for (size_t k = 0; k < cnt; k++)
            if (a[k] < 0 || a[k] >= hi) return false;
        return true;
    };
    if (d->n_bend < 0 || (d->n_bend && (!d->bend_offsets || d->bend_offsets[d->n_bend] < 0))) return false;
    return ok(d->tri_inds, 3 * (size_t)std::max(d->n_tri, 0), nd) && ok(d->tet_inds, 4 * (size_t)std::max(d->n_tet, 0), nd) &&
           ok(d->bend_inds, d->n_bend ? (size_t)d->bend_offsets[d->n_bend] : 0, nd) &&
           ok(d->pin_inds, (size_t)std::max(d->n_pin, 0), nd) && ok(d->surf_tris, 3 * (size_t)std::max(d->n_surf_tri, 0), n) &&
           ok(d->surf_edges, 2 * (size_t)std::max(d->n_surf_edge, 0), n) &&
           ok(d->surf_verts, (size_t)std::max(d->n_surf_vert, 0), n);
}

// Morton order (21 bits per axis) of the dynamic vertices' rest positions, ties by index;
// static vertices keep their indices.
void morton_order(const AdmmB200Desc* d, std::vector<int>& perm, std::vector<int>& iperm) {
    const int n = d->n_vert, nd = d->n_dyn;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < nd; i++)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], d->x0[3 * i + k]);
            hi[k] = std::max(hi[k], d->x0[3 * i + k]);
        }
    const double ext = std::max({(double)hi[0] - lo[0], (double)hi[1] - lo[1], (double)hi[2] - lo[2], 1e-30});
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    std::vector<std::pair<uint64_t, int>> key(nd);
    for (int i = 0; i < nd; i++) {
        uint64_t c[3];
        for (int k = 0; k < 3; k++) {
            const double t = ((double)d->x0[3 * i + k] - lo[k]) / ext;
            c[k] = (uint64_t)std::min(2097151.0, std::max(0.0, t * 2097151.0));
        }
        key[i] = {spread(c[0]) | spread(c[1]) << 1 | spread(c[2]) << 2, i};
    }
    std::sort(key.begin(), key.end());
    perm.resize(n);
    iperm.resize(n);
    for (int i = 0; i < nd; i++) perm[i] = key[i].second;
    for (int i = nd; i < n; i++) perm[i] = i;
    for (int i = 0; i < n; i++) iperm[perm[i]] = i;
}

// A copy of the description with the dynamic vertices in the order perm.
void renumber(const AdmmB200Desc* in, const std::vector<int>& perm, const std::vector<int>& iperm, RenumberedDesc& r) {
    const int n = in->n_vert;
    r.d = *in;
    auto per_vertex = [&](const float* a, std::vector<float>& out, int width) -> const float* {
        if (!a) return nullptr;
        out.resize((size_t)width * n);
        for (int i = 0; i < n; i++)
            for (int k = 0; k < width; k++) out[(size_t)width * i + k] = a[(size_t)width * perm[i] + k];
        return out.data();
    };
    auto map_idx = [&](const int32_t* a, size_t cnt, std::vector<int32_t>& out) -> const int32_t* {
        if (!a) return nullptr;
        out.resize(cnt);
        for (size_t k = 0; k < cnt; k++) out[k] = iperm[a[k]];
        return out.data();
    };
    r.d.x0 = per_vertex(in->x0, r.x0, 3);
    r.d.v0 = per_vertex(in->v0, r.v0, 3);
    r.d.mass = per_vertex(in->mass, r.mass, 1);
    r.d.contact_w = per_vertex(in->contact_w, r.cw, 1);
    r.d.vert_mu = per_vertex(in->vert_mu, r.vmu, 1);
    if (in->is_fixed) {
        r.fixed.resize(n);
        for (int i = 0; i < n; i++) r.fixed[i] = in->is_fixed[perm[i]];
        r.d.is_fixed = r.fixed.data();
    }
    r.d.tri_inds = map_idx(in->tri_inds, 3 * (size_t)in->n_tri, r.tri);
    r.d.tet_inds = map_idx(in->tet_inds, 4 * (size_t)in->n_tet, r.tet);
    r.d.bend_inds = map_idx(in->bend_inds, in->n_bend ? (size_t)in->bend_offsets[in->n_bend] : 0, r.bend);
    r.d.pin_inds = map_idx(in->pin_inds, (size_t)in->n_pin, r.pin);
    r.d.surf_tris = map_idx(in->surf_tris, 3 * (size_t)in->n_surf_tri, r.st);
    r.d.surf_edges = map_idx(in->surf_edges, 2 * (size_t)in->n_surf_edge, r.se);
    if (in->surf_verts) {
        map_idx(in->surf_verts, (size_t)in->n_surf_vert, r.sv);
        std::sort(r.sv.begin(), r.sv.end());  // the detection's vertex queries in the new order
        r.d.surf_verts = r.sv.data();
    }
}

extern "C" {

const char* admm_b200_errstr(int code) {
    const int k = -code;
    if (k < 0 || k >= (int)(sizeof(kErrStr) / sizeof(kErrStr[0]))) return "unknown status";
    return kErrStr[k];
}

const char* admm_b200_last_error(const AdmmB200* h) { return h ? h->last_error.c_str() : "null handle"; }

int admm_b200_create(const AdmmB200Desc* desc, int device, AdmmB200** out) {
    if (!desc || !out) return ADMM_ERR_INVALID;
    *out = nullptr;
    AdmmB200* h = new (std::nothrow) AdmmB200;
    if (!h) return ADMM_ERR_OOM;
    const char* env = std::getenv("ADMM_B200_RENUMBER");
    const bool want = desc->abi_version == ADMM_B200_ABI_VERSION && desc->backend_semantics == 0 && desc->x0 &&
                      desc->mass && env && env[0] == '1' && env[1] == '\0' && indices_in_range(desc);
    RenumberedDesc rd;
    if (want) {
        morton_order(desc, h->perm, h->iperm);
        renumber(desc, h->perm, h->iperm, rd);
    }
    int rc = create_impl(want ? &rd.d : desc, device, h);
    if (rc == ADMM_OK && want) {
        rc = dupload(h, &h->d_perm, h->perm.data(), h->perm.size());
        if (rc == ADMM_OK) {
            // the global matrix in the caller's order, for admm_b200_system
            const HostCsr& A = h->hostA;
            const int nd = h->s.nd;
            HostCsr& C = h->hostA_caller;
            C.start.assign(nd + 1, 0);
            for (int j = 0; j < nd; j++) {
                const int i = h->iperm[j];
                std::vector<std::pair<int, double>> e;
                for (int k = A.start[i]; k < A.start[i + 1]; k++) e.push_back({h->perm[A.col[k]], A.val[k]});
                std::sort(e.begin(), e.end());
                for (auto& kv : e) {
                    C.col.push_back(kv.first);
                    C.val.push_back(kv.second);
                }
                C.start[j + 1] = (int)C.col.size();
            }
        }
    }
    if (rc != ADMM_OK) {
        static thread_local std::string err;
        err = h->last_error;
        fprintf(stderr, "admm_b200_create: %s (%s)\n", admm_b200_errstr(rc), err.c_str());
        admm_b200_destroy(h);
        return rc;
    }
    *out = h;
    return ADMM_OK;
}

void admm_b200_destroy(AdmmB200* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
    if (h->fail_host) cudaFreeHost(h->fail_host);
    for (void* p : h->allocs)
        if (p) cudaFree(p);
    for (auto e : h->prof_ev) cudaEventDestroy(e);
    for (auto e : h->probe_ev) cudaEventDestroy(e);
    for (auto e : h->pev) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->body_stream) cudaStreamDestroy(h->body_stream);
    if (h->if_stream) cudaStreamDestroy(h->if_stream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);

    delete h;
}

int admm_b200_step_async(AdmmB200* h, int n_steps) {
    if (!h) return ADMM_ERR_INVALID;
    if (n_steps < 0) return fail(h, ADMM_ERR_INVALID, "n_steps");
    CK(cudaSetDevice(h->device));
    if (h->profiling) {
        // eager, one substep at a time so that every event pair can be read back
        CK(cudaEventRecord(h->ev0, h->stream));
        for (int k = 0; k < n_steps; k++) {
            h->prof_used = 0;
            TRY(run_substep_eager(h));
            CK(cudaStreamSynchronize(h->stream));
            TRY(accumulate_timers(h));
        }
        CK(cudaEventRecord(h->ev1, h->stream));
        h->frame += n_steps;
        return ADMM_OK;
    }
    TRY(build_step_graph(h));
    CK(cudaEventRecord(h->ev0, h->stream));
    for (int k = 0; k < n_steps; k++) TRY(launch_substep(h));
    CK(cudaEventRecord(h->ev1, h->stream));
    h->frame += n_steps;
    return ADMM_OK;
}

int admm_b200_sync(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

int admm_b200_step(AdmmB200* h, int n_steps, AdmmStepStats* stats) {
    if (!h) return ADMM_ERR_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    TRY(admm_b200_step_async(h, n_steps));
    CK(cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->last_ms = n_steps > 0 ? ms / n_steps : 0.f;
    if (!h->profiling) TRY(accumulate_timers(h));
    int status = ADMM_OK;
    TRY(read_err_flags(h, &status));
    int nc = 0;
    CK(cudaMemcpy(&nc, h->s.nc, sizeof(int), cudaMemcpyDeviceToHost));
    h->peak = std::max(h->peak, nc);
    h->last_iters = h->admm_max_iter;
    if (h->residual_tol > 0.f) CK(cudaMemcpy(&h->last_iters, h->s.done, sizeof(int), cudaMemcpyDeviceToHost));
    if (stats) {
        double r[4];
        CK(cudaMemcpy(r, h->s.res, sizeof(r), cudaMemcpyDeviceToHost));
        stats->frame = h->frame;
        stats->step_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() /
                         (n_steps > 0 ? n_steps : 1);
        stats->n_contacts = nc;
        stats->admm_iters = h->last_iters;
        const double sc = r[2] > 0.0 ? std::sqrt(r[2]) : 1.0;
        stats->primal_residual = std::sqrt(r[0]) / sc;
        stats->dual_residual = std::sqrt(r[1]) / sc;
        stats->status = status;
        stats->peak_contacts = h->peak;
    }
    return status;
}

int admm_b200_set_state(AdmmB200* h, const float* x, const float* v, int n) {
    if (!h || !x) return ADMM_ERR_INVALID;
    if (n != h->s.n) return fail(h, ADMM_ERR_INVALID, "n must equal n_vert");
    CK(cudaSetDevice(h->device));
    std::vector<float4> hx(n), hv(n, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int i = 0; i < n; i++) {
        const int c = caller_of(h, i);
        hx[i] = pack(x + 3 * c);
        if (v) hv[i] = pack(v + 3 * c);
    }
    CK(cudaStreamSynchronize(h->stream));
    return upload_state(h, hx, hv);
}

int admm_b200_get_state(AdmmB200* h, float* x, float* v, int n) {
    if (!h) return ADMM_ERR_INVALID;
    if (n != h->s.n) return fail(h, ADMM_ERR_INVALID, "n must equal n_vert");
    CK(cudaSetDevice(h->device));
    std::vector<float4> tmp(n);
    CK(cudaStreamSynchronize(h->stream));
    if (x) {
        CK(cudaMemcpy(tmp.data(), h->s.x0, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++) {
            const int c = caller_of(h, i);
            x[3 * c] = tmp[i].x; x[3 * c + 1] = tmp[i].y; x[3 * c + 2] = tmp[i].z;
        }
    }
    if (v) {
        CK(cudaMemcpy(tmp.data(), h->s.v, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++) {
            const int c = caller_of(h, i);
            v[3 * c] = tmp[i].x; v[3 * c + 1] = tmp[i].y; v[3 * c + 2] = tmp[i].z;
        }
    }
    return ADMM_OK;
}

int admm_b200_reset(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    DevScene& s = h->s;
    CK(cudaMemset(s.ue, 0, sizeof(float4) * s.m));
    CK(cudaMemset(s.z, 0, sizeof(float4) * s.m));
    CK(cudaMemset(s.y, 0, sizeof(float4) * s.m));
    CK(cudaMemset(s.uc, 0, sizeof(float4) * s.nd));
    CK(cudaMemset(s.p, 0, sizeof(float4) * s.n));
    CK(cudaMemset(s.rc, 0, sizeof(float4) * s.cap));
    CK(cudaMemset(s.nc, 0, sizeof(int)));
    CK(cudaMemset(s.err, 0, sizeof(int) * 4));
    h->frame = 0;
    h->peak = 0;
    TRY(upload_state(h, h->x_init, h->v_init));
    return anim_init(h);
}

int admm_b200_set_rigid_track(AdmmB200* h, int32_t v0, int32_t v1, int32_t n_frames, const float* pos,
                              const float* quat) {
    if (!h || !pos || !quat) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    TRY(check_track_range(h, v0, v1, n_frames));
    if (n_frames < 3) return fail(h, ADMM_ERR_INVALID, "a rigid track needs at least 3 frames");
    std::vector<float4> p(n_frames), q(n_frames), rest(h->x_init.begin() + v0, h->x_init.begin() + v1);
    for (int f = 0; f < n_frames; f++) {
        p[f] = make_float4(pos[3 * f], pos[3 * f + 1], pos[3 * f + 2], 0.f);
        q[f] = make_float4(quat[4 * f], quat[4 * f + 1], quat[4 * f + 2], quat[4 * f + 3]);
    }
    TrackDev t;
    t.kind = 0;
    t.v0 = v0;
    t.v1 = v1;
    t.n_frames = n_frames;
    float4 *dp, *dq, *dr;
    TRY(dupload(h, &dp, p.data(), p.size()));
    TRY(dupload(h, &dq, q.data(), q.size()));
    TRY(dupload(h, &dr, rest.data(), rest.size()));
    t.pos = dp;
    t.quat = dq;
    t.rest = dr;
    return add_track(h, t);
}

int admm_b200_set_point_track(AdmmB200* h, int32_t v0, int32_t v1, int32_t n_frames, const float* points,
                              const float* rot9, const float* translate3, float scale) {
    if (!h || !points || !rot9 || !translate3) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    TRY(check_track_range(h, v0, v1, n_frames));
    const size_t nv = (size_t)(v1 - v0);
    std::vector<float4> pts(nv * (size_t)n_frames);
    for (size_t k = 0; k < pts.size(); k++) pts[k] = make_float4(points[3 * k], points[3 * k + 1], points[3 * k + 2], 0.f);
    TrackDev t;
    t.kind = 1;
    t.v0 = v0;
    t.v1 = v1;
    t.n_frames = n_frames;
    for (int k = 0; k < 9; k++) t.rot[k] = rot9[k];
    for (int k = 0; k < 3; k++) t.trans[k] = translate3[k];
    t.scale = scale;
    float4* dp;
    TRY(dupload(h, &dp, pts.data(), pts.size()));
    t.pts = dp;
    return add_track(h, t);
}

int admm_b200_clear_tracks(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    for (auto& t : h->tracks) {
        dfree(h, const_cast<float4*>(t.pos));
        dfree(h, const_cast<float4*>(t.quat));
        dfree(h, const_cast<float4*>(t.rest));
        dfree(h, const_cast<float4*>(t.pts));
    }
    h->tracks.clear();
    return anim_publish(h);
}

int admm_b200_device_state(AdmmB200* h, void** x, void** v) {
    if (!h) return ADMM_ERR_INVALID;
    if (x) *x = h->s.x0;
    if (v) *v = h->s.v;
    return ADMM_OK;
}

int admm_b200_vertex_order(AdmmB200* h, int32_t* order, int n) {
    if (!h || !order) return ADMM_ERR_INVALID;
    if (n != h->s.n) return fail(h, ADMM_ERR_INVALID, "n must equal n_vert");
    for (int i = 0; i < n; i++) order[i] = caller_of(h, i);
    return ADMM_OK;
}

int admm_b200_read_buffer(AdmmB200* h, int which, float* out, int n) {
    if (!h || !out) return ADMM_ERR_INVALID;
    int rows = 0;
    float4* p = buffer_ptr(h, which, &rows);
    if (!p || n != rows) return fail(h, ADMM_ERR_INVALID, "buffer id or row count");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<float4> tmp(rows);
    CK(cudaMemcpy(tmp.data(), p, sizeof(float4) * rows, cudaMemcpyDeviceToHost));
    const bool pv = per_vertex_buffer(which);
    for (int i = 0; i < rows; i++) {
        const int c = pv ? caller_of(h, i) : i;
        out[3 * c] = tmp[i].x; out[3 * c + 1] = tmp[i].y; out[3 * c + 2] = tmp[i].z;
    }
    return ADMM_OK;
}

int admm_b200_write_buffer(AdmmB200* h, int which, const float* in, int n) {
    if (!h || !in) return ADMM_ERR_INVALID;
    int rows = 0;
    float4* p = buffer_ptr(h, which, &rows);
    if (!p || n != rows) return fail(h, ADMM_ERR_INVALID, "buffer id or row count");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<float4> tmp(rows);
    const bool pv = per_vertex_buffer(which);
    for (int i = 0; i < rows; i++) tmp[i] = pack(in + 3 * (pv ? caller_of(h, i) : i));
    CK(cudaMemcpy(p, tmp.data(), sizeof(float4) * rows, cudaMemcpyHostToDevice));
    if (which == ADMM_BUF_Z || which == ADMM_BUF_UE) {
        // keep y = z - Ue consistent for the right-hand side
        std::vector<float4> z(h->s.m), ue(h->s.m);
        CK(cudaMemcpy(z.data(), h->s.z, sizeof(float4) * h->s.m, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ue.data(), h->s.ue, sizeof(float4) * h->s.m, cudaMemcpyDeviceToHost));
        for (int i = 0; i < h->s.m; i++) z[i] = make_float4(z[i].x - ue[i].x, z[i].y - ue[i].y, z[i].z - ue[i].z, 0.f);
        CK(cudaMemcpy(h->s.y, z.data(), sizeof(float4) * h->s.m, cudaMemcpyHostToDevice));
    }
    return ADMM_OK;
}

int admm_b200_local_step(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    enqueue_local(h, LOCAL_PROX);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

int admm_b200_global_step(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    enqueue_global(h, false, true);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

int admm_b200_jacobi(AdmmB200* h, int sweeps) {
    if (!h || sweeps < 0) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    enqueue_jacobi(h, sweeps);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

int admm_b200_pre_integration(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    LAUNCH(k_pre_integration, blocks(h->s.n, kVertThreads), kVertThreads, h->s);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

int admm_b200_detect(AdmmB200* h, int* count) {
    if (!h) return ADMM_ERR_INVALID;
    if (!h->s.contact) return fail(h, ADMM_ERR_STATE, "contact disabled in the description");
    CK(cudaSetDevice(h->device));
    enqueue_dcd(h);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    int raw = 0, nc = 0;
    CK(cudaMemcpy(&raw, h->s.nc_raw, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&nc, h->s.nc, sizeof(int), cudaMemcpyDeviceToHost));
    h->peak = std::max(h->peak, nc);
    h->detected = true;
    if (count) *count = raw;
    int status = ADMM_OK;
    TRY(read_err_flags(h, &status));
    return status;
}

int admm_b200_detect_host(AdmmB200* h, const float* x, int n, int* count) {
    if (!h || !x) return ADMM_ERR_INVALID;
    if (n != h->s.n) return fail(h, ADMM_ERR_INVALID, "n must equal n_vert");
    CK(cudaSetDevice(h->device));
    std::vector<float4> hx(n);
    for (int i = 0; i < n; i++) hx[i] = pack(x + 3 * caller_of(h, i));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(h->s.x, hx.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    return admm_b200_detect(h, count);
}

int admm_b200_contact_step(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    if (!h->s.contact || !h->detected) return fail(h, ADMM_ERR_STATE, "contact_step needs a detection first");
    CK(cudaSetDevice(h->device));
    h->cstream = h->stream;
    TRY(enqueue_contact(h, false));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return ADMM_OK;
}

int admm_b200_contacts(AdmmB200* h, int32_t* pairs, float* bary4, float* normal3, float* point3, float* gap,
                       int cap, int* count) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    int nc = 0;
    CK(cudaMemcpy(&nc, h->s.nc, sizeof(int), cudaMemcpyDeviceToHost));
    if (count) *count = nc;
    const int k = std::min(nc, std::max(cap, 0));
    if (k == 0) return ADMM_OK;
    if (pairs) {
        CK(cudaMemcpy(pairs, h->s.pairs, sizeof(int4) * k, cudaMemcpyDeviceToHost));
        if (!h->perm.empty())
            for (int i = 0; i < 4 * k; i++) pairs[i] = h->perm[pairs[i]];
    }
    std::vector<float4> tmp(k);
    if (bary4) CK(cudaMemcpy(bary4, h->s.bary, sizeof(float4) * k, cudaMemcpyDeviceToHost));
    if (normal3 || gap) {
        CK(cudaMemcpy(tmp.data(), h->s.nrm, sizeof(float4) * k, cudaMemcpyDeviceToHost));
        for (int i = 0; i < k; i++) {
            if (normal3) { normal3[3 * i] = tmp[i].x; normal3[3 * i + 1] = tmp[i].y; normal3[3 * i + 2] = tmp[i].z; }
            if (gap) gap[i] = tmp[i].w;
        }
    }
    if (point3) {
        CK(cudaMemcpy(tmp.data(), h->s.point, sizeof(float4) * k, cudaMemcpyDeviceToHost));
        for (int i = 0; i < k; i++) { point3[3 * i] = tmp[i].x; point3[3 * i + 1] = tmp[i].y; point3[3 * i + 2] = tmp[i].z; }
    }
    return ADMM_OK;
}

int admm_b200_contact_count(AdmmB200* h, int* count) {
    if (!h || !count) return ADMM_ERR_INVALID;
    return admm_b200_contacts(h, nullptr, nullptr, nullptr, nullptr, nullptr, 0, count);
}

int admm_b200_max_slots(AdmmB200* h, int* slots) {
    if (!h || !slots) return ADMM_ERR_INVALID;
    *slots = h->s.cap;
    return ADMM_OK;
}

int admm_b200_peak_contact_count(AdmmB200* h, int* peak) {
    if (!h || !peak) return ADMM_ERR_INVALID;
    *peak = h->peak;
    return ADMM_OK;
}

int admm_b200_clear_contacts(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemset(h->s.nc, 0, sizeof(int)));
    CK(cudaMemset(h->s.nc_raw, 0, sizeof(int)));
    return ADMM_OK;
}

int admm_b200_residuals(AdmmB200* h, double* primal, double* dual) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    double r[4];
    CK(cudaMemcpy(r, h->s.res, sizeof(r), cudaMemcpyDeviceToHost));
    const double sc = r[2] > 0.0 ? std::sqrt(r[2]) : 1.0;
    if (primal) *primal = std::sqrt(r[0]) / sc;
    if (dual) *dual = std::sqrt(r[1]) / sc;
    return ADMM_OK;
}

int admm_b200_last_step_device_ms(AdmmB200* h, float* ms) {
    if (!h || !ms) return ADMM_ERR_INVALID;
    *ms = h->last_ms;
    return ADMM_OK;
}

int admm_b200_set_profiling(AdmmB200* h, int enabled) {
    if (!h) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (enabled && h->prof_ev.empty()) {
        h->prof_ev.resize(kMaxProfEvents);
        h->prof_phase.assign(kMaxProfEvents / 2, 0);
        for (auto& e : h->prof_ev) CK(cudaEventCreate(&e));
    }
    h->profiling = enabled != 0;
    h->prof_used = 0;
    return ADMM_OK;
}

int admm_b200_step_host(AdmmB200* h, const float* x_in, const float* v_in, float* x_out, float* v_out, int n) {
    if (!h || !x_in) return ADMM_ERR_INVALID;
    if (n != h->s.n) return fail(h, ADMM_ERR_INVALID, "n must equal n_vert");
    CK(cudaSetDevice(h->device));
    if (!h->stage) TRY(dalloc(h, &h->stage, (size_t)6 * n));
    TRY(build_step_graph(h));
    const size_t bytes = sizeof(float) * 3 * (size_t)n;
    CK(cudaMemcpyAsync(h->stage, x_in, bytes, cudaMemcpyHostToDevice, h->stream));
    if (v_in) CK(cudaMemcpyAsync(h->stage + 3 * (size_t)n, v_in, bytes, cudaMemcpyHostToDevice, h->stream));
    k_unpack_state<<<blocks(n, 256), 256, 0, h->stream>>>(h->s, h->stage, v_in ? 1 : 0, h->d_perm);
    TRY(launch_substep(h));
    k_pack_state<<<blocks(n, 256), 256, 0, h->stream>>>(h->s, h->stage, h->d_perm);
    if (x_out) CK(cudaMemcpyAsync(x_out, h->stage, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (v_out) CK(cudaMemcpyAsync(v_out, h->stage + 3 * (size_t)n, bytes, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->frame += 1;
    int status = ADMM_OK;
    TRY(read_err_flags(h, &status));
    return status;
}

int admm_b200_phase_times(AdmmB200* h, double* ms, int64_t* launches, int n_phases) {
    if (!h) return ADMM_ERR_INVALID;
    for (int k = 0; k < n_phases && k < ADMM_NUM_PHASES; k++) {
        if (ms) ms[k] = h->phase_ms[k];
        if (launches) launches[k] = h->phase_launches[k];
        h->phase_ms[k] = 0.0;
        h->phase_launches[k] = 0;
    }
    return ADMM_OK;
}

int admm_b200_set_probe(AdmmB200* h, int kernel_class) {
    if (!h || kernel_class < 0 || (kernel_class > ADMM_KERNEL_DCD_EE && kernel_class != ADMM_PROBE_PHASES))
        return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (h->step_exec) {
        cudaGraphExecDestroy(h->step_exec);
        h->step_exec = nullptr;
    }
    h->probe_kernel = kernel_class;
    h->probe_ms = 0.0;
    h->probe_n = 0;
    return ADMM_OK;
}

int admm_b200_probe_time(AdmmB200* h, double* mean_ms, int64_t* count) {
    if (!h) return ADMM_ERR_INVALID;
    if (mean_ms) *mean_ms = h->probe_n ? h->probe_ms / (double)h->probe_n : 0.0;
    if (count) *count = h->probe_n;
    h->probe_ms = 0.0;
    h->probe_n = 0;
    return ADMM_OK;
}

int admm_b200_tuning(AdmmB200* h, int* lanes_a, int* lanes_r, float* ms_a, float* ms_r) {
    if (!h) return ADMM_ERR_INVALID;
    if (lanes_a) *lanes_a = h->tune_lanes_a;
    if (lanes_r) *lanes_r = h->tune_lanes_r;
    if (ms_a) *ms_a = h->tune_ms_a;
    if (ms_r) *ms_r = h->tune_ms_r;
    return ADMM_OK;
}

int admm_b200_system(AdmmB200* h, int32_t* start, int32_t* col, float* val, float* diag) {
    if (!h) return ADMM_ERR_INVALID;
    const HostCsr& A = h->perm.empty() ? h->hostA : h->hostA_caller;
    const int nnz = (int)A.col.size();
    if (!start) return nnz;
    if (!col || !val || !diag) return ADMM_ERR_INVALID;
    for (size_t i = 0; i < A.start.size(); i++) start[i] = A.start[i];
    for (int k = 0; k < nnz; k++) {
        col[k] = A.col[k];
        val[k] = (float)A.val[k];
    }
    for (size_t i = 0; i < h->hostAdiag.size(); i++) diag[caller_of(h, (int)i)] = h->hostAdiag[i];
    return nnz;
}

int admm_b200_set_preconditioner(AdmmB200* h, const float* blocks9, int nd) {
    if (!h || !blocks9) return ADMM_ERR_INVALID;
    if (nd != h->s.nd) return fail(h, ADMM_ERR_INVALID, "nd must equal n_dyn");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (!h->pcg_blocks) TRY(dalloc(h, &h->pcg_blocks, 9 * (size_t)nd));
    std::vector<float> bl(9 * (size_t)nd);
    for (int i = 0; i < nd; i++)
        for (int k = 0; k < 9; k++) bl[9 * (size_t)i + k] = blocks9[9 * (size_t)caller_of(h, i) + k];
    CK(cudaMemcpy(h->pcg_blocks, bl.data(), sizeof(float) * 9 * (size_t)nd, cudaMemcpyHostToDevice));
    // the step graph holds the preconditioner pointer: capture it again
    if (h->step_exec) {
        cudaGraphExecDestroy(h->step_exec);
        h->step_exec = nullptr;
    }
    return ADMM_OK;
}

int admm_b200_set_learned(AdmmB200* h, int sweeps, const float* omega, const float* beta, const float* m,
                          const float* theta, int nd) {
    if (!h || !omega || !beta) return ADMM_ERR_INVALID;
    if (sweeps < 1 || sweeps > kLearnMaxSweeps) return fail(h, ADMM_ERR_INVALID, "sweeps must be 1..32");
    if (nd != h->s.nd) return fail(h, ADMM_ERR_INVALID, "nd must equal n_dyn");
    for (int k = 0; k < sweeps; k++)
        if (!std::isfinite(omega[k]) || !std::isfinite(beta[k])) return fail(h, ADMM_ERR_INVALID, "omega/beta");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<float> mv(nd), th(nd, 0.f);
    for (int i = 0; i < nd; i++) {
        const int c = caller_of(h, i);
        mv[i] = m ? m[c] : 1.f / h->hostAdiag[i];
        if (theta) th[i] = theta[c];
        if (!std::isfinite(mv[i]) || !std::isfinite(th[i])) return fail(h, ADMM_ERR_INVALID, "m/theta");
    }
    CK(cudaMemcpy(const_cast<float*>(h->learn.minv), mv.data(), sizeof(float) * nd, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(const_cast<float*>(h->learn.theta), th.data(), sizeof(float) * nd, cudaMemcpyHostToDevice));
    h->learn_sweeps = sweeps;
    h->learn_omega.assign(omega, omega + sweeps);
    h->learn_beta.assign(beta, beta + sweeps);
    h->learn_beta[0] = 0.f;  // the first sweep has no previous iterate
    // the coefficients are kernel arguments of the step graph: capture it again
    if (h->step_exec) {
        cudaGraphExecDestroy(h->step_exec);
        h->step_exec = nullptr;
    }
    return ADMM_OK;
}

int admm_b200_learned_stats(AdmmB200* h, int64_t* out4) {
    if (!h || !out4) return ADMM_ERR_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    unsigned long long d[2] = {0, 0};
    CK(cudaMemcpy(d, h->learn.stats, sizeof(d), cudaMemcpyDeviceToHost));
    out4[0] = h->learn_substeps;
    out4[1] = (int64_t)d[1];  // every failed solve was replaced by the plain one
    out4[2] = (int64_t)d[0];
    out4[3] = (int64_t)d[1];
    return ADMM_OK;
}

int admm_b200_record_global(AdmmB200* h, int iteration, float* b, float* x_cur, float* x_last, int nd) {
    if (!h || !b || !x_cur || !x_last) return ADMM_ERR_INVALID;
    if (nd != h->s.nd) return fail(h, ADMM_ERR_INVALID, "nd must equal n_dyn");
    if (iteration < 1 || iteration >= h->admm_max_iter) return fail(h, ADMM_ERR_INVALID, "iteration must be 1..admm_max_iter-1");
    CK(cudaSetDevice(h->device));
    if (!h->rec_b) {
        TRY(dalloc(h, &h->rec_b, nd));
        TRY(dalloc(h, &h->rec_cur, nd));
        TRY(dalloc(h, &h->rec_last, nd));
    }
    h->rec_target = iteration;
    h->rec_count = 0;
    const bool prof = h->profiling;
    h->profiling = false;
    const int rc = run_substep_eager(h);
    h->profiling = prof;
    const int recorded = h->rec_count;
    h->rec_target = -1;
    TRY(rc);
    CK(cudaStreamSynchronize(h->stream));
    h->frame += 1;
    if (recorded <= iteration) return fail(h, ADMM_ERR_STATE, "the substep ended before the recorded iteration");
    std::vector<float4> t(nd);
    float* outs[3] = {b, x_cur, x_last};
    float4* srcs[3] = {h->rec_b, h->rec_cur, h->rec_last};
    for (int k = 0; k < 3; k++) {
        CK(cudaMemcpy(t.data(), srcs[k], sizeof(float4) * nd, cudaMemcpyDeviceToHost));
        for (int i = 0; i < nd; i++) {
            const int c = caller_of(h, i);
            outs[k][3 * c] = t[i].x;
            outs[k][3 * c + 1] = t[i].y;
            outs[k][3 * c + 2] = t[i].z;
        }
    }
    return ADMM_OK;
}

int admm_b200_global_mode(AdmmB200* h, int* persistent, int* blocks, float* ms_sweeps, float* ms_persist) {
    if (!h) return ADMM_ERR_INVALID;
    if (persistent) *persistent = h->persist ? 1 : h->tiled ? 3 : 0;
    if (blocks) *blocks = h->persist ? h->pp.blocks : 0;
    if (ms_sweeps) *ms_sweeps = h->tune_ms_sweeps;
    if (ms_persist) *ms_persist = h->tune_ms_persist;
    return ADMM_OK;
}

int admm_b200_kernels_fallback(AdmmB200* h, int* n) {
    if (!h || !n) return ADMM_ERR_INVALID;
    TRY(build_step_graph(h));
    *n = h->global_solver == 3 ? h->kernels_fallback : 0;
    return ADMM_OK;
}

int admm_b200_kernels_per_step(AdmmB200* h, int* n) {
    if (!h || !n) return ADMM_ERR_INVALID;
    TRY(build_step_graph(h));
    *n = h->kernels_per_step;
    // residual-tolerance mode: the first chunk runs outside the conditional node
    if (h->residual_tol > 0.f && h->chunk > 0) {
        const int it = h->last_iters > 0 ? h->last_iters : h->chunk;
        *n += h->kernels_body * (it / h->chunk - 1);
    }
    return ADMM_OK;
}

}  // extern "C"
