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
// in two registers per lane up to 64 keys, else read back from vtmp.  Static
// vertices are sorted too: their lists are read by no gather, but k_contact_p
// and the incidence entries cover all positions.
constexpr int kRankSortRegs = 64;

// The vertices with contacts, ascending: tv[tpos[i]] = i for vcnt[i] > 0
// (tpos = exclusive scan of vcnt != 0, *ntv = their number).
__global__ void __launch_bounds__(kContactThreads) k_contact_touched(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s.n && s.vcnt[i] > 0) s.tv[s.tpos[i]] = i;
}

// One warp per vertex with contacts (grid-stride over the touched list).
__global__ void __launch_bounds__(kContactThreads) k_contact_sort_lists(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int lane = threadIdx.x & 31;
    const int ntv = *s.ntv;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntv; t += (gridDim.x * blockDim.x) >> 5) {
        const int i = s.tv[t];
        const int b = s.vstart[i], e = s.vstart[i + 1], L = e - b;
        if (L <= kRankSortRegs) {
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
        const float sc = s.eps + (b.x * b.x * s.cwinv[q.x] * (float)s.vcnt[q.x] +
                                  b.y * b.y * s.cwinv[q.y] * (float)s.vcnt[q.y] +
                                  b.z * b.z * s.cwinv[q.z] * (float)s.vcnt[q.z] +
                                  b.w * b.w * s.cwinv[q.w] * (float)s.vcnt[q.w]);
        s.gamma[c] = make_float4(b.x / (sc * s.cw[q.x]), b.y / (sc * s.cw[q.y]), b.z / (sc * s.cw[q.z]),
                                 b.w / (sc * s.cw[q.w]));
        const float4 nr = s.nrm[c];
        const float k = s.dt_inv * nr.w;
        s.kc[c] = f4(k * nr.x * s.gam, k * nr.y * s.gam, k * nr.z * s.gam);
        s.rc[c] = f4(0.f, 0.f, 0.f);
        s.du[c] = f4(0.f, 0.f, 0.f);
        float mu = s.mu;
        if (s.vmu) mu = s.vmu[q.x < s.nd ? q.x : q.y < s.nd ? q.y : q.z < s.nd ? q.z : q.w];
        s.cmu[c] = mu;
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

// Projection of u = sum_k bary_k p_k + K_c onto the friction cone for contact c
// with accumulated correction r: returns du (the caller sets r_c = r + du).
ADMM_DEV float4 friction_cone_du(const DevScene& s, int c, float ux, float uy, float uz, float4 r) {
    const float4 n = s.nrm[c];
    const float sx = ux - r.x, sy = uy - r.y, sz = uz - r.z;
    float uN = n.x * sx + n.y * sy + n.z * sz;
    float tx = sx - uN * n.x, ty = sy - uN * n.y, tz = sz - uN * n.z;
    if (uN < 0.f) {
        const float tau = sqrtf(tx * tx + ty * ty + tz * tz);
        const float alpha = -s.cmu[c] * uN;
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

// u_c = sum_k bary_k p_k + K_c for contact c from the p values of its four vertices.
ADMM_DEV void contact_u_of(const DevScene& s, int c, float4 p0, float4 p1, float4 p2, float4 p3, float& ux,
                           float& uy, float& uz) {
    const float4 b = s.bary[c];
    const float4 kc = s.kc[c];
    ux = b.x * p0.x + b.y * p1.x + b.z * p2.x + b.w * p3.x;
    uy = b.x * p0.y + b.y * p1.y + b.z * p2.y + b.w * p3.y;
    uz = b.x * p0.z + b.y * p1.z + b.z * p2.z + b.w * p3.z;
    ux = ux + kc.x;
    uy = uy + kc.y;
    uz = uz + kc.z;
}

// u_c from the p values in `p`.
ADMM_DEV void contact_u(const DevScene& s, int c, const float4* __restrict__ p, float& ux, float& uy, float& uz) {
    const int4 q = s.pairs[c];
    contact_u_of(s, c, p[q.x], p[q.y], p[q.z], p[q.w], ux, uy, uz);
}

__global__ void __launch_bounds__(kContactThreads) k_contact_du(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int nc = ccount(s);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        float ux, uy, uz;
        contact_u(s, c, s.p, ux, uy, uz);
        const float4 r = s.rc[c];
        const float4 d = friction_cone_du(s, c, ux, uy, uz, r);
        s.du[c] = d;
        s.rc[c] = f4(r.x + d.x, r.y + d.y, r.z + d.z);
    }
}

// p_i = p_src_i + sum_c Gamma_c,i du_c over the incidence list of vertex i
// (update_p, contact_solver.cu:381-399) into s.p, kGatherLanes lanes per vertex
// with contacts (grid-stride over the touched list; static vertices skipped).
__global__ void __launch_bounds__(kContactThreads) k_contact_gather(DevScene s, const float4* __restrict__ p_src,
                                                                   const float4* __restrict__ du) {
    ADMM_PDL_PROLOGUE();
    const int sub = threadIdx.x % kGatherLanes;
    const unsigned gmask = 0xffu << (threadIdx.x & 31 & ~(kGatherLanes - 1));
    const int ntv = *s.ntv;
    const int g0 = (blockIdx.x * blockDim.x + threadIdx.x) / kGatherLanes;
    const int gs = gridDim.x * blockDim.x / kGatherLanes;
    for (int t = g0; t < ntv; t += gs) {  // uniform per group
        const int i = s.tv[t];
        if (i >= s.nd) continue;
        const float4 acc = gather_group(s, du, s.vstart[i], s.vstart[i + 1], sub, gmask);
        if (sub == 0) {
            float4 p = p_src[i];
            p.x += acc.x;
            p.y += acc.y;
            p.z += acc.z;
            s.p[i] = p;
        }
    }
}

// One projection pass fused with the gather of the previous one, a warp per
// contact: the four lane groups of 8 rebuild p of the contact's four vertices
// from p_old and the previous pass's du_old (the same sums, in the same order,
// as k_contact_gather), the first contact of each vertex's incidence list
// stores that p into p_new for the next pass, and lane 0 projects the contact
// (du_new, r_c += du) from those p.  Static vertices keep p in s.p.  Replaces
// a gather + projection pair of launches with one launch and one round trip.
__global__ void __launch_bounds__(kContactThreads) k_contact_pass(DevScene s, const float4* __restrict__ p_old,
                                                                 float4* __restrict__ p_new,
                                                                 const float4* __restrict__ du_old,
                                                                 float4* __restrict__ du_new) {
    ADMM_PDL_PROLOGUE();
    const int lane = threadIdx.x & 31, grp = lane >> 3, sub = lane & 7;
    const unsigned gmask = 0xffu << (lane & ~7);
    const int nc = ccount(s);
    const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, ws = (gridDim.x * blockDim.x) >> 5;
    for (int c = w0; c < nc; c += ws) {  // uniform per warp
        const int4 q = s.pairs[c];
        const int v = grp == 0 ? q.x : grp == 1 ? q.y : grp == 2 ? q.z : q.w;
        float4 pv;
        if (v >= s.nd) {  // uniform per group
            pv = s.p[v];
        } else {
            const int b = s.vstart[v];
            const float4 acc = gather_group(s, du_old, b, s.vstart[v + 1], sub, gmask);
            pv = p_old[v];
            pv.x += acc.x;
            pv.y += acc.y;
            pv.z += acc.z;
            if (sub == 0 && __float_as_int(s.ginc[b].x) == c) p_new[v] = pv;
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
            contact_u_of(s, c, p0, p1, p2, p3, ux, uy, uz);
            const float4 r = s.rc[c];
            const float4 d = friction_cone_du(s, c, ux, uy, uz, r);
            du_new[c] = d;
            s.rc[c] = f4(r.x + d.x, r.y + d.y, r.z + d.z);
        }
    }
}

}  // namespace admm
