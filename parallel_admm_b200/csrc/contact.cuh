// contact.cuh -- frictional contact in velocity space (GPU semantics of the
// reference, contact_solver.cu:90-431), on a deterministic vertex -> contact
// incidence list.
#pragma once
#include "common.cuh"
#include "scene_dev.cuh"

namespace admm {

constexpr int kContactThreads = 256;

ADMM_DEV int ccount(const DevScene& s) { return *s.nc; }

ADMM_DEV float comp(float4 v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

// per-vertex contact counts over all four vertices (updateContactCounts,
// contact_solver.cu:90-101)
__global__ void __launch_bounds__(kContactThreads) k_contact_count(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int nc = ccount(s);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int4 q = s.pairs[c];
        atomicAdd(&s.vcnt[q.x], 1);
        atomicAdd(&s.vcnt[q.y], 1);
        atomicAdd(&s.vcnt[q.z], 1);
        atomicAdd(&s.vcnt[q.w], 1);
    }
}

// incidence slots (compute_Scc_kernel's CSR fill, contact_solver.cu:210-223)
__global__ void __launch_bounds__(kContactThreads) k_contact_fill(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int nc = ccount(s);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int4 q = s.pairs[c];
        const int v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int pos = atomicAdd(&s.vfill[v[k]], 1);
            s.vtmp[s.vstart[v[k]] + pos] = 4 * c + k;
        }
    }
}

// Sort each vertex's incidence list by (contact, slot) so the gathers below
// sum in a fixed order (the reference's order depends on atomics, F13).  The
// fill leaves the lists unsorted in vtmp; one warp per vertex writes each key
// to vlist at its rank (the keys are distinct), counted against the list held
// in two registers per lane up to 64 keys, else read back from vtmp.  The lists
// of static vertices are read by no gather: they are copied unsorted (a static
// ground under an impact holds thousands of entries, and the quadratic sort of
// those lists dominated the detection), so that vlist and the incidence entries
// still cover every position.
constexpr int kRankSortRegs = 64;

// The vertices with contacts, ascending: tv[tpos[i]] = i for vcnt[i] > 0
// (tpos = exclusive scan of vcnt != 0, *ntv = their number), and beside it the
// vertex with its incidence-list bounds (tvr), which the gather loads in one
// round trip.
__global__ void __launch_bounds__(kContactThreads) k_contact_touched(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s.n && s.vcnt[i] > 0) {
        const int t = s.tpos[i];
        s.tv[t] = i;
        s.tvr[t] = make_int4(i, s.vstart[i], s.vstart[i + 1], 0);
    }
}

// One warp per vertex with contacts (grid-stride over the touched list).
__global__ void __launch_bounds__(kContactThreads) k_contact_sort_lists(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int lane = threadIdx.x & 31;
    const int ntv = *s.ntv;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntv; t += (gridDim.x * blockDim.x) >> 5) {
        const int i = s.tv[t];
        const int b = s.vstart[i], e = s.vstart[i + 1], L = e - b;
        if (i >= s.nd) {
            for (int m = lane; m < L; m += 32) s.vlist[b + m] = s.vtmp[b + m];
        } else if (L <= kRankSortRegs) {
            const int k0 = lane < L ? s.vtmp[b + lane] : 0x7fffffff;
            const int k1 = lane + 32 < L ? s.vtmp[b + 32 + lane] : 0x7fffffff;
            int r0 = 0, r1 = 0;
            for (int j = 0; j < L; j++) {
                const int kj = __shfl_sync(0xffffffffu, j < 32 ? k0 : k1, j & 31);
                r0 += kj < k0;
                r1 += kj < k1;
            }
            if (lane < L) s.vlist[b + r0] = k0;
            if (lane + 32 < L) s.vlist[b + r1] = k1;
        } else {
            for (int m = lane; m < L; m += 32) {
                const int key = s.vtmp[b + m];
                int r = 0;
                for (int j = 0; j < L; j++) r += s.vtmp[b + j] < key;
                s.vlist[b + r] = key;
            }
        }
    }
}

// S_c, Gamma_c, K_c, r_c = 0 (compute_Scc_kernel, contact_solver.cu:188-227;
// the fills at 240-243).
__global__ void __launch_bounds__(kContactThreads) k_contact_scc(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int nc = ccount(s);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int4 q = s.pairs[c];
        const float4 b = s.bary[c];
        // the CPU backend (compute_Scc, admm_impl_cpu.cpp:361-380) leaves out the
        // per-vertex contact counts and sets Gamma of static vertices to zero
        const float c0 = s.cpu_backend ? 1.f : (float)s.vcnt[q.x], c1 = s.cpu_backend ? 1.f : (float)s.vcnt[q.y];
        const float c2 = s.cpu_backend ? 1.f : (float)s.vcnt[q.z], c3 = s.cpu_backend ? 1.f : (float)s.vcnt[q.w];
        const float sc = s.eps + (b.x * b.x * s.cwinv[q.x] * c0 + b.y * b.y * s.cwinv[q.y] * c1 +
                                  b.z * b.z * s.cwinv[q.z] * c2 + b.w * b.w * s.cwinv[q.w] * c3);
        float4 gm = make_float4(b.x / (sc * s.cw[q.x]), b.y / (sc * s.cw[q.y]), b.z / (sc * s.cw[q.z]),
                                b.w / (sc * s.cw[q.w]));
        if (s.cpu_backend) {
            if (s.cw[q.x] > 1e7f) gm.x = 0.f;
            if (s.cw[q.y] > 1e7f) gm.y = 0.f;
            if (s.cw[q.z] > 1e7f) gm.z = 0.f;
            if (s.cw[q.w] > 1e7f) gm.w = 0.f;
        }
        s.gamma[c] = gm;
        const float4 nr = s.nrm[c];
        const float k = s.dt_inv * nr.w;
        s.kc[c] = f4(k * nr.x * s.gam, k * nr.y * s.gam, k * nr.z * s.gam);
        s.rc[c] = f4(0.f, 0.f, 0.f);
        s.du[c] = f4(0.f, 0.f, 0.f);
        float mu = s.mu;
        if (s.vmu) mu = s.vmu[q.x < s.nd ? q.x : q.y < s.nd ? q.y : q.z < s.nd ? q.z : q.w];
        s.cmu[c] = mu;
        const int v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; k++) s.cinc[4 * c + k] = make_int4(v[k], s.vstart[v[k]], s.vstart[v[k] + 1], 0);
    }
}

// Friction-cone projection of contact c (get_delta_u_kernel, contact_solver.cu:337-379).
// Incidence entries in list order: (contact, Gamma_c,i) for every position of
// the sorted lists, so that a gather needs no further indirection.
__global__ void __launch_bounds__(kContactThreads) k_contact_incidence(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int n4 = 4 * ccount(s);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n4; k += gridDim.x * blockDim.x) {
        const int slot = s.vlist[k];
        const int c = slot >> 2;
        s.ginc[k] = make_float2(__int_as_float(c), comp(s.gamma[c], slot & 3));
    }
}

// Sum of Gamma_c,i v_c over the incidence entries [b, e) of one vertex by the
// kGatherLanes lanes of a group: lane l takes entries b+l, b+l+G, ...; the
// partial sums are combined by xor shuffles (a fixed order), every lane gets
// the total.
constexpr int kGatherLanes = 8;

ADMM_DEV float4 gather_group(const DevScene& s, const float4* __restrict__ v, int b, int e, int sub, unsigned gmask) {
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (int k = b + sub; k < e; k += kGatherLanes) {
        const float2 gi = s.ginc[k];
        const float4 d = v[__float_as_int(gi.x)];
        ax = fmaf(d.x, gi.y, ax);
        ay = fmaf(d.y, gi.y, ay);
        az = fmaf(d.z, gi.y, az);
    }
#pragma unroll
    for (int o = kGatherLanes / 2; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(gmask, ax, o, kGatherLanes);
        ay += __shfl_xor_sync(gmask, ay, o, kGatherLanes);
        az += __shfl_xor_sync(gmask, az, o, kGatherLanes);
    }
    return f4(ax, ay, az);
}

// Projection of u = sum_k bary_k p_k + K_c onto the friction cone of normal n
// and coefficient mu with accumulated correction r: returns du (the caller sets
// r_c = r + du).
ADMM_DEV float4 cone_du(float4 n, float mu, float ux, float uy, float uz, float4 r) {
    const float sx = ux - r.x, sy = uy - r.y, sz = uz - r.z;
    float uN = n.x * sx + n.y * sy + n.z * sz;
    float tx = sx - uN * n.x, ty = sy - uN * n.y, tz = sz - uN * n.z;
    if (uN < 0.f) {
        const float tau = sqrtf(tx * tx + ty * ty + tz * tz);
        const float alpha = -mu * uN;
        uN = 0.f;
        if (tau <= alpha) {
            tx = ty = tz = 0.f;
        } else {
            const float f = 1.f - alpha / tau;
            tx *= f; ty *= f; tz *= f;
        }
    }
    return f4(uN * n.x + tx - ux, uN * n.y + ty - uy, uN * n.z + tz - uz);
}

// u = sum_k bary_k p_k + K_c from the p values of the contact's four vertices.
ADMM_DEV void contact_u_bk(float4 b, float4 kc, float4 p0, float4 p1, float4 p2, float4 p3, float& ux, float& uy,
                           float& uz) {
    ux = b.x * p0.x + b.y * p1.x + b.z * p2.x + b.w * p3.x;
    uy = b.x * p0.y + b.y * p1.y + b.z * p2.y + b.w * p3.y;
    uz = b.x * p0.z + b.y * p1.z + b.z * p2.z + b.w * p3.z;
    ux = ux + kc.x;
    uy = uy + kc.y;
    uz = uz + kc.z;
}

// What only a detection writes about contact c (vertices, barycentric weights,
// K_c, normal, friction coefficient), read through L2 (ld.global.cg): the
// projection kernels load it before their dependency wait, when no line that
// L1 may hold from before the detection must be read.
struct ContactRec {
    int4 q;
    float4 b, kc, n;
    float mu;
};

ADMM_DEV ContactRec contact_rec(const DevScene& s, int c) {
    ContactRec r;
    r.q = __ldcg(&s.pairs[c]);
    r.b = __ldcg(&s.bary[c]);
    r.kc = __ldcg(&s.kc[c]);
    r.n = __ldcg(&s.nrm[c]);
    r.mu = __ldcg(&s.cmu[c]);
    return r;
}

// First projection of an ADMM iteration, a thread per contact, from s.p into
// s.du (get_delta_u_kernel, contact_solver.cu:337-379).  k_contact_p before it
// waits before it triggers, so the detection has completed when this kernel
// starts: the contact records are loaded before the wait, only p and r_c after.
__global__ void __launch_bounds__(kContactThreads) k_contact_du(DevScene s) {
    const int c0 = blockIdx.x * blockDim.x + threadIdx.x, cs = gridDim.x * blockDim.x;
    const int nc = __ldcg(s.nc);
    ContactRec R0 = {};
    if (c0 < nc) R0 = contact_rec(s, c0);
    ADMM_PDL_WAIT_THEN_TRIGGER();
    for (int c = c0; c < nc; c += cs) {
        const ContactRec R = c == c0 ? R0 : contact_rec(s, c);
        const float4 r = s.rc[c];
        float ux, uy, uz;
        contact_u_bk(R.b, R.kc, s.p[R.q.x], s.p[R.q.y], s.p[R.q.z], s.p[R.q.w], ux, uy, uz);
        const float4 d = cone_du(R.n, R.mu, ux, uy, uz, r);
        s.du[c] = d;
        s.rc[c] = f4(r.x + d.x, r.y + d.y, r.z + d.z);
    }
}

// p_i = p_src_i + sum_c Gamma_c,i du_c over the incidence list of vertex i
// (update_p, contact_solver.cu:381-399) into s.p, kGatherLanes lanes per vertex
// with contacts (grid-stride over the touched list; static vertices skipped).
// The pass before it waits before it triggers: the touched list, the list
// bounds and the first two incidence entries of each lane (detection data) are
// loaded before the wait.
__global__ void __launch_bounds__(kContactThreads) k_contact_gather(DevScene s, const float4* __restrict__ p_src,
                                                                   const float4* __restrict__ du) {
    ADMM_PDL_TRIGGER();
    const int sub = threadIdx.x % kGatherLanes;
    const unsigned gmask = 0xffu << (threadIdx.x & 31 & ~(kGatherLanes - 1));
    const int ntv = __ldcg(s.ntv);
    const int g0 = (blockIdx.x * blockDim.x + threadIdx.x) / kGatherLanes;
    const int gs = gridDim.x * blockDim.x / kGatherLanes;
    int i0 = -1, b0 = 0, e0 = 0;
    float2 gi0[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    if (g0 < s.n) {  // tvr has n entries: loaded beside ntv, used below ntv only
        const int4 r = __ldcg(&s.tvr[g0]);
        if (g0 < ntv && r.x < s.nd) {
            i0 = r.x;
            b0 = r.y;
            e0 = r.z;
#pragma unroll
            for (int j = 0; j < 2; j++)
                if (b0 + sub + j * kGatherLanes < e0) gi0[j] = __ldcg(&s.ginc[b0 + sub + j * kGatherLanes]);
        }
    }
    ADMM_PDL_WAIT();
    for (int t = g0; t < ntv; t += gs) {  // uniform per group
        const bool first = t == g0;
        const int4 r = first ? make_int4(i0, b0, e0, 0) : s.tvr[t];
        const int i = first ? i0 : r.x;
        if (i < 0 || i >= s.nd) continue;
        const int b = r.y, e = r.z;
        float4 p = p_src[i];
        float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int k = b + sub + j * kGatherLanes;
            if (k < e) {
                const float2 gi = first ? gi0[j] : s.ginc[k];
                const float4 d = du[__float_as_int(gi.x)];
                ax = fmaf(d.x, gi.y, ax);
                ay = fmaf(d.y, gi.y, ay);
                az = fmaf(d.z, gi.y, az);
            }
        }
        for (int k = b + sub + 2 * kGatherLanes; k < e; k += kGatherLanes) {
            const float2 gi = s.ginc[k];
            const float4 d = du[__float_as_int(gi.x)];
            ax = fmaf(d.x, gi.y, ax);
            ay = fmaf(d.y, gi.y, ay);
            az = fmaf(d.z, gi.y, az);
        }
#pragma unroll
        for (int o = kGatherLanes / 2; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(gmask, ax, o, kGatherLanes);
            ay += __shfl_xor_sync(gmask, ay, o, kGatherLanes);
            az += __shfl_xor_sync(gmask, az, o, kGatherLanes);
        }
        if (sub == 0) {
            p.x += ax;
            p.y += ay;
            p.z += az;
            s.p[i] = p;
        }
    }
}

// What a projection pass reads of the detection for one contact and one lane
// group (one of the contact's four vertices): the contact record, the vertex,
// its incidence-list bounds and the lane's first entry, or p of a static
// vertex (set before the contact step).  All through L2 (see ContactRec).
struct PassRec {
    ContactRec r;
    int v, b, e;
    float2 gi;
    float4 pst;
};

ADMM_DEV PassRec pass_rec(const DevScene& s, int c, int grp, int sub) {
    PassRec P;
    P.r = contact_rec(s, c);
    const int4 ci = __ldcg(&s.cinc[4 * c + grp]);  // beside the record, not after it
    P.v = ci.x;
    P.b = ci.y;
    P.e = ci.z;
    P.gi = make_float2(0.f, 0.f);
    P.pst = f4(0.f, 0.f, 0.f);
    if (P.v >= s.nd) P.pst = __ldcg(&s.p[P.v]);
    else if (P.b + sub < P.e) P.gi = __ldcg(&s.ginc[P.b + sub]);
    return P;
}

// The pass for contact c, from its PassRec P.
ADMM_DEV void pass_contact(const DevScene& s, int c, const PassRec& P, int lane, int sub, unsigned gmask,
                           const float4* __restrict__ p_old, float4* __restrict__ p_new,
                           const float4* __restrict__ du_old, float4* __restrict__ du_new) {
    const float4 r = lane == 0 ? s.rc[c] : f4(0.f, 0.f, 0.f);  // issued beside the gathers
    float4 pv;
    if (P.v >= s.nd) {  // uniform per group
        pv = P.pst;
    } else {
        float ax = 0.f, ay = 0.f, az = 0.f;
        const float4 po = p_old[P.v];
        if (P.b + sub < P.e) {
            const float4 d = du_old[__float_as_int(P.gi.x)];
            ax = fmaf(d.x, P.gi.y, ax);
            ay = fmaf(d.y, P.gi.y, ay);
            az = fmaf(d.z, P.gi.y, az);
        }
        for (int k = P.b + sub + kGatherLanes; k < P.e; k += kGatherLanes) {
            const float2 gi = s.ginc[k];
            const float4 d = du_old[__float_as_int(gi.x)];
            ax = fmaf(d.x, gi.y, ax);
            ay = fmaf(d.y, gi.y, ay);
            az = fmaf(d.z, gi.y, az);
        }
#pragma unroll
        for (int o = kGatherLanes / 2; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(gmask, ax, o, kGatherLanes);
            ay += __shfl_xor_sync(gmask, ay, o, kGatherLanes);
            az += __shfl_xor_sync(gmask, az, o, kGatherLanes);
        }
        pv = po;
        pv.x += ax;
        pv.y += ay;
        pv.z += az;
        if (sub == 0 && __float_as_int(P.gi.x) == c) p_new[P.v] = pv;
    }
    const float4 p0 = f4(__shfl_sync(0xffffffffu, pv.x, 0), __shfl_sync(0xffffffffu, pv.y, 0),
                         __shfl_sync(0xffffffffu, pv.z, 0));
    const float4 p1 = f4(__shfl_sync(0xffffffffu, pv.x, 8), __shfl_sync(0xffffffffu, pv.y, 8),
                         __shfl_sync(0xffffffffu, pv.z, 8));
    const float4 p2 = f4(__shfl_sync(0xffffffffu, pv.x, 16), __shfl_sync(0xffffffffu, pv.y, 16),
                         __shfl_sync(0xffffffffu, pv.z, 16));
    const float4 p3 = f4(__shfl_sync(0xffffffffu, pv.x, 24), __shfl_sync(0xffffffffu, pv.y, 24),
                         __shfl_sync(0xffffffffu, pv.z, 24));
    if (lane == 0) {
        float ux, uy, uz;
        contact_u_bk(P.r.b, P.r.kc, p0, p1, p2, p3, ux, uy, uz);
        const float4 d = cone_du(P.r.n, P.r.mu, ux, uy, uz, r);
        du_new[c] = d;
        s.rc[c] = f4(r.x + d.x, r.y + d.y, r.z + d.z);
    }
}

// One projection pass fused with the gather of the previous one, a warp per
// contact: the four lane groups of 8 rebuild p of the contact's four vertices
// from p_old and the previous pass's du_old (the same sums, in the same order,
// as k_contact_gather), the first contact of each vertex's incidence list
// stores that p into p_new for the next pass, and lane 0 projects the contact
// (du_new, r_c += du) from those p.  Static vertices keep p in s.p.  Replaces
// a gather + projection pair of launches with one launch and one round trip.
// The kernel before it (k_contact_du or the previous pass) waits before it
// triggers, so the detection data of the warp's first contact (PassRec) is
// loaded before the wait; after it only du_old, p_old and r_c.
__global__ void __launch_bounds__(kContactThreads) k_contact_pass(DevScene s, const float4* __restrict__ p_old,
                                                                    float4* __restrict__ p_new,
                                                                 const float4* __restrict__ du_old,
                                                                 float4* __restrict__ du_new) {
    const int lane = threadIdx.x & 31, grp = lane >> 3, sub = lane & 7;
    const unsigned gmask = 0xffu << (lane & ~7);
    const int nc = __ldcg(s.nc);
    const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, ws = (gridDim.x * blockDim.x) >> 5;
    PassRec P0 = {};
    if (w0 < s.cap) P0 = pass_rec(s, w0, grp, sub);  // in bounds; beside nc, used below nc only
    ADMM_PDL_WAIT_THEN_TRIGGER();
    if (w0 < nc) pass_contact(s, w0, P0, lane, sub, gmask, p_old, p_new, du_old, du_new);
    for (int c = w0 + ws; c < nc; c += ws)  // uniform per warp
        pass_contact(s, c, pass_rec(s, c, grp, sub), lane, sub, gmask, p_old, p_new, du_old, du_new);
}

// The CPU backend's contact projection after the warm start: `passes` serial
// Gauss-Seidel sweeps over the contact list in its order, each contact projected
// from the current p and its update scattered into p at once
// (_project_feasible_plain / _project_one_contact, admm_impl_cpu.cpp:390-448).
// One thread: the order is the algorithm.
__global__ void k_contact_gs_serial(DevScene s, int passes) {
    ADMM_PDL_PROLOGUE();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nc = *s.nc;
    for (int it = 0; it < passes; it++)
        for (int c = 0; c < nc; c++) {
            const int4 q = s.pairs[c];
            const float4 b = s.bary[c], kc = s.kc[c], g = s.gamma[c], r = s.rc[c];
            float ux, uy, uz;
            contact_u_bk(b, kc, s.p[q.x], s.p[q.y], s.p[q.z], s.p[q.w], ux, uy, uz);
            const float4 d = cone_du(s.nrm[c], s.cmu[c], ux, uy, uz, r);
            s.rc[c] = f4(r.x + d.x, r.y + d.y, r.z + d.z);
            const int v[4] = {q.x, q.y, q.z, q.w};
            const float gg[4] = {g.x, g.y, g.z, g.w};
            for (int k = 0; k < 4; k++) {
                if (v[k] >= s.nd) continue;
                float4 pv = s.p[v[k]];
                pv.x = fmaf(gg[k], d.x, pv.x);
                pv.y = fmaf(gg[k], d.y, pv.y);
                pv.z = fmaf(gg[k], d.z, pv.z);
                s.p[v[k]] = pv;
            }
        }
}

}  // namespace admm
