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
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "admm_b200.h"
#include "contact.cuh"
#include "kernels.cuh"
#include "lbvh.cuh"
#include "scan_sort.cuh"
#include "setup.hpp"

using namespace admm;

struct AdmmB200 {
    int device = 0;
    cudaStream_t stream = nullptr;
    DevScene s;
    std::vector<void*> allocs;
    std::string last_error;
    // scene scalars
    int admm_max_iter = 0, dcd_interval = 1, gs_iter = 0, jac_iter = 0;
    int tet_blocks = 0, tri_blocks = 0, bend_blocks = 0, pin_blocks = 0;
    int contact_grid = 1;
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
                         "call out of order"};

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
    return ADMM_OK;
}

// ------------------------------ enqueue helpers -----------------------------
#define LAUNCH(kernel, grid, block, ...)                                   \
    do {                                                                   \
        kernel<<<(grid), (block), 0, h->stream>>>(__VA_ARGS__);            \
        h->launch_counter++;                                               \
    } while (0)

void enqueue_build(AdmmB200* h, BvhDev& t, const int* elems, int stride, bool tri) {
    const int n = t.n;
    if (n <= 0) return;
    if (tri) LAUNCH(k_elem_boxes<3>, blocks(n, 256), 256, h->s.x, elems, stride, n, t);
    else LAUNCH(k_elem_boxes<2>, blocks(n, 256), 256, h->s.x, elems, stride, n, t);
    LAUNCH(k_morton, blocks(n, 256), 256, t);
    if (n > 1) {
        radix_sort(t.keys, t.vals, t.keys_alt, t.vals_alt, n, 64, h->hist, h->s.scan_tmp, h->stream);
        h->launch_counter += 8 * 5;
    }
    LAUNCH(k_karras, blocks(n, 256), 256, t);
    LAUNCH(k_refit, blocks(n, 256), 256, t);
}

// DCD + contact conversion + incidence lists + S_c / Gamma / K_c, all on device.
void enqueue_dcd(AdmmB200* h) {
    DevScene& s = h->s;
    LAUNCH(k_scene_init, 1, 32, s.bf, s.be);
    enqueue_build(h, s.bf, (const int*)s.st, 4, true);
    enqueue_build(h, s.be, (const int*)s.se, 2, false);
    const int nq = s.nsv + s.nse;
    if (s.nsv > 0) LAUNCH(k_dcd_vf<false>, blocks(s.nsv, 128), 128, s);
    if (s.nse > 0) LAUNCH(k_dcd_ee<false>, blocks(s.nse, 128), 128, s);
    if (nq > 0) {
        exclusive_scan(s.qcount, s.qoff, nq, s.scan_tmp, s.nc_raw, h->stream);
        h->launch_counter += 3;
    } else {
        cudaMemsetAsync(s.nc_raw, 0, sizeof(int), h->stream);
    }
    LAUNCH(k_set_count, 1, 1, s);
    if (s.nsv > 0) LAUNCH(k_dcd_vf<true>, blocks(s.nsv, 128), 128, s);
    if (s.nse > 0) LAUNCH(k_dcd_ee<true>, blocks(s.nse, 128), 128, s);
    cudaMemsetAsync(s.vcnt, 0, sizeof(int) * s.n, h->stream);
    cudaMemsetAsync(s.vfill, 0, sizeof(int) * s.n, h->stream);
    LAUNCH(k_contact_count, h->contact_grid, kContactThreads, s);
    exclusive_scan(s.vcnt, s.vstart, s.n, s.scan_tmp, s.vstart + s.n, h->stream);
    h->launch_counter += 3;
    LAUNCH(k_contact_fill, h->contact_grid, kContactThreads, s);
    LAUNCH(k_contact_sort_lists, blocks(s.nd, kContactThreads), kContactThreads, s);
    LAUNCH(k_contact_scc, h->contact_grid, kContactThreads, s);
}

void enqueue_local(AdmmB200* h, int mode) {
    const int g = h->tet_blocks + h->tri_blocks + h->bend_blocks + h->pin_blocks;
    if (mode == LOCAL_PROX)
        LAUNCH(k_local<LOCAL_PROX>, g, kLocalThreads, h->s, h->tet_blocks, h->tri_blocks, h->bend_blocks);
    else if (mode == (LOCAL_PROX | LOCAL_DUAL))
        LAUNCH(k_local<LOCAL_PROX | LOCAL_DUAL>, g, kLocalThreads, h->s, h->tet_blocks, h->tri_blocks, h->bend_blocks);
    else
        LAUNCH(k_local<LOCAL_DUAL>, g, kLocalThreads, h->s, h->tet_blocks, h->tri_blocks, h->bend_blocks);
}

void enqueue_contact(AdmmB200* h, bool dual) {
    DevScene& s = h->s;
    const int vb = blocks(s.nd, kVertThreads);
    if (dual) LAUNCH((k_contact_p<true, true>), vb, kVertThreads, s);
    else LAUNCH((k_contact_p<false, true>), vb, kVertThreads, s);
    for (int g = 0; g < h->gs_iter; g++) {
        LAUNCH(k_contact_du, h->contact_grid, kContactThreads, s);
        LAUNCH(k_contact_gather, blocks(s.nd, kContactThreads), kContactThreads, s);
    }
}

void enqueue_jacobi(AdmmB200* h, int sweeps) {
    DevScene& s = h->s;
    const int vb = blocks(s.nd, kVertThreads);
    if (sweeps <= 0) return;
    if (sweeps == 1) {
        LAUNCH(k_jacobi, vb, kVertThreads, s, s.x, s.jac[0]);
        LAUNCH(k_copy_dyn, vb, kVertThreads, s, s.jac[0], s.x);
        return;
    }
    for (int k = 0; k < sweeps; k++) {
        const float4* src = k == 0 ? s.x : s.jac[(k - 1) & 1];
        float4* dst = k == sweeps - 1 ? s.x : s.jac[k & 1];
        LAUNCH(k_jacobi, vb, kVertThreads, s, src, dst);
    }
}

void enqueue_global(AdmmB200* h, bool save_prev) {
    const int vb = blocks(h->s.nd, kVertThreads);
    if (save_prev) LAUNCH(k_rhs<true>, vb, kVertThreads, h->s);
    else LAUNCH(k_rhs<false>, vb, kVertThreads, h->s);
    enqueue_jacobi(h, h->jac_iter);
}

void enqueue_residual(AdmmB200* h) {
    DevScene& s = h->s;
    cudaMemsetAsync(s.res, 0, sizeof(double) * 4, h->stream);
    const int vb = blocks(s.nd, kLocalThreads);
    const int g = h->tet_blocks + h->tri_blocks + h->bend_blocks + h->pin_blocks + vb;
    LAUNCH(k_residual, g, kLocalThreads, s, h->tet_blocks, h->tri_blocks, h->bend_blocks, h->pin_blocks);
}

// One substep (ADMMImplGPU::step).  The residual of the last iteration is kept.
void enqueue_step(AdmmB200* h) {
    DevScene& s = h->s;
    LAUNCH(k_pre_integration, blocks(s.n, kVertThreads), kVertThreads, s);
    if (!h->warmstart_ue) cudaMemsetAsync(s.ue, 0, sizeof(float4) * s.m, h->stream);
    if (!h->warmstart_uc) cudaMemsetAsync(s.uc, 0, sizeof(float4) * s.nd, h->stream);
    for (int it = 0; it < h->admm_max_iter; it++) {
        const bool first = it == 0, last = it == h->admm_max_iter - 1;
        if (s.contact && it % h->dcd_interval == 0) enqueue_dcd(h);
        enqueue_local(h, first ? LOCAL_PROX : (LOCAL_PROX | LOCAL_DUAL));
        if (s.contact) enqueue_contact(h, !first);
        enqueue_global(h, last);
        if (last) enqueue_residual(h);
    }
    if (h->admm_max_iter > 0) enqueue_local(h, LOCAL_DUAL);
    LAUNCH(k_vertex_final, blocks(s.n, kVertThreads), kVertThreads, s);
}

int build_step_graph(AdmmB200* h) {
    if (h->step_exec) return ADMM_OK;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->launch_counter = 0;
    enqueue_step(h);
    h->kernels_per_step = h->launch_counter;
    CK(cudaStreamEndCapture(h->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&h->step_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(h, ADMM_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return ADMM_OK;
}

float4 pack(const float* p) { return make_float4(p[0], p[1], p[2], 0.f); }

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
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return fail(h, ADMM_ERR_NO_DEVICE, "no CUDA device");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(h, ADMM_ERR_NO_DEVICE, "device is not sm_100 (Blackwell B200)");
    CK(cudaSetDevice(device));
    h->device = device;

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
    // matrices
    {
        int *p, *c; float* v; float* dg;
        TRY(dupload(h, &p, as.A.ptr.data(), as.A.ptr.size()));
        TRY(dupload(h, &c, as.A.col.data(), as.A.col.size()));
        TRY(dupload(h, &v, as.A.val.data(), as.A.val.size()));
        TRY(dupload(h, &dg, as.a_diag.data(), nd));
        s.A.rows = nd; s.A.nslices = as.A.nslices; s.A.ptr = p; s.A.col = c; s.A.val = v; s.a_diag = dg;
        TRY(dupload(h, &p, as.R.ptr.data(), as.R.ptr.size()));
        TRY(dupload(h, &c, as.R.col.data(), as.R.col.size()));
        TRY(dupload(h, &v, as.R.val.data(), as.R.val.size()));
        s.R.rows = nd; s.R.nslices = as.R.nslices; s.R.ptr = p; s.R.col = c; s.R.val = v;
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
    TRY(dalloc(h, &s.du, s.cap));
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
    const int scan_n = std::max(std::max(scan_tiles(hist_n), scan_tiles(n + 1)), scan_tiles(s.nsv + s.nse + 1)) + 4;
    TRY(dalloc(h, &s.scan_tmp, scan_n));
    TRY(dalloc(h, &s.res, 4));
    TRY(dalloc(h, &s.done, 4));
    h->contact_grid = std::max(1, std::min(blocks(s.cap, kContactThreads), 148 * 8));

    h->tet_blocks = s.ntet ? blocks(s.ntet, kLocalThreads) : 0;
    h->tri_blocks = s.ntri ? blocks(s.ntri, kLocalThreads) : 0;
    h->bend_blocks = s.nbend ? blocks(s.nbend, kLocalThreads) : 0;
    h->pin_blocks = s.npin ? blocks(s.npin, kLocalThreads) : 0;
    if (h->tet_blocks + h->tri_blocks + h->bend_blocks + h->pin_blocks == 0) return fail(h, ADMM_ERR_INVALID, "no constraints");

    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    TRY(upload_state(h, h->x_init, h->v_init));
    return ADMM_OK;
}

int read_err_flags(AdmmB200* h, int* status) {
    int e[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(e, h->s.err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e[0] || e[1] || e[2]) CK(cudaMemset(h->s.err, 0, sizeof(int) * 4));
    *status = e[0] ? ADMM_ERR_CONTACT_OVERFLOW : e[1] ? ADMM_ERR_STACK_OVERFLOW : e[2] ? ADMM_ERR_NAN : ADMM_OK;
    return ADMM_OK;
}

}  // namespace

// ================================ C ABI =====================================
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
    const int rc = create_impl(desc, device, h);
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
    for (void* p : h->allocs) cudaFree(p);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int admm_b200_step_async(AdmmB200* h, int n_steps) {
    if (!h) return ADMM_ERR_INVALID;
    if (n_steps < 0) return fail(h, ADMM_ERR_INVALID, "n_steps");
    CK(cudaSetDevice(h->device));
    TRY(build_step_graph(h));
    CK(cudaEventRecord(h->ev0, h->stream));
    for (int k = 0; k < n_steps; k++) CK(cudaGraphLaunch(h->step_exec, h->stream));
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
    int status = ADMM_OK;
    TRY(read_err_flags(h, &status));
    int nc = 0;
    CK(cudaMemcpy(&nc, h->s.nc, sizeof(int), cudaMemcpyDeviceToHost));
    h->peak = std::max(h->peak, nc);
    if (stats) {
        double r[4];
        CK(cudaMemcpy(r, h->s.res, sizeof(r), cudaMemcpyDeviceToHost));
        stats->frame = h->frame;
        stats->step_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() /
                         (n_steps > 0 ? n_steps : 1);
        stats->n_contacts = nc;
        stats->admm_iters = h->admm_max_iter;
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
        hx[i] = pack(x + 3 * i);
        if (v) hv[i] = pack(v + 3 * i);
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
        for (int i = 0; i < n; i++) { x[3 * i] = tmp[i].x; x[3 * i + 1] = tmp[i].y; x[3 * i + 2] = tmp[i].z; }
    }
    if (v) {
        CK(cudaMemcpy(tmp.data(), h->s.v, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++) { v[3 * i] = tmp[i].x; v[3 * i + 1] = tmp[i].y; v[3 * i + 2] = tmp[i].z; }
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
    return upload_state(h, h->x_init, h->v_init);
}

int admm_b200_device_state(AdmmB200* h, void** x, void** v) {
    if (!h) return ADMM_ERR_INVALID;
    if (x) *x = h->s.x0;
    if (v) *v = h->s.v;
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
    for (int i = 0; i < rows; i++) { out[3 * i] = tmp[i].x; out[3 * i + 1] = tmp[i].y; out[3 * i + 2] = tmp[i].z; }
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
    for (int i = 0; i < rows; i++) tmp[i] = pack(in + 3 * i);
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
    enqueue_global(h, false);
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
    for (int i = 0; i < n; i++) hx[i] = pack(x + 3 * i);
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(h->s.x, hx.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    return admm_b200_detect(h, count);
}

int admm_b200_contact_step(AdmmB200* h) {
    if (!h) return ADMM_ERR_INVALID;
    if (!h->s.contact || !h->detected) return fail(h, ADMM_ERR_STATE, "contact_step needs a detection first");
    CK(cudaSetDevice(h->device));
    enqueue_contact(h, false);
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
    if (pairs) CK(cudaMemcpy(pairs, h->s.pairs, sizeof(int4) * k, cudaMemcpyDeviceToHost));
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
    (void)enabled;
    return ADMM_OK;
}

int admm_b200_kernels_per_step(AdmmB200* h, int* n) {
    if (!h || !n) return ADMM_ERR_INVALID;
    TRY(build_step_graph(h));
    *n = h->kernels_per_step;
    return ADMM_OK;
}

}  // extern "C"
