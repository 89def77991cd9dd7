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
            s.vlist[s.vstart[v[k]] + pos] = 4 * c + k;
        }
    }
}

// Sort each vertex's incidence list by (contact, slot) so the gather below
// sums in a fixed order (the reference's order depends on atomics, F13).
__global__ void __launch_bounds__(kContactThreads) k_contact_sort_lists(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.nd) return;
    const int b = s.vstart[i], e = s.vstart[i + 1];
    for (int k = b + 1; k < e; k++) {
        const int key = s.vlist[k];
        int j = k - 1;
        while (j >= b && s.vlist[j] > key) {
            s.vlist[j + 1] = s.vlist[j];
            j--;
        }
        s.vlist[j + 1] = key;
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
    }
}

// Friction-cone projection of contact c (get_delta_u_kernel, contact_solver.cu:337-379).
// Projection of u = sum_k bary_k p_k + K_c onto the friction cone for contact c
// with accumulated correction r: returns du (the caller sets r_c = r + du).
ADMM_DEV float4 friction_cone_du(const DevScene& s, int c, float ux, float uy, float uz, float4 r) {
    const float4 n = s.nrm[c];
    const float sx = ux - r.x, sy = uy - r.y, sz = uz - r.z;
    float uN = n.x * sx + n.y * sy + n.z * sz;
    float tx = sx - uN * n.x, ty = sy - uN * n.y, tz = sz - uN * n.z;
    if (uN < 0.f) {
        const float tau = sqrtf(tx * tx + ty * ty + tz * tz);
        const float alpha = -s.mu * uN;
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

// u_c = sum_k bary_k p_k + K_c for contact c, from the p values in `p`.
ADMM_DEV void contact_u(const DevScene& s, int c, const float4* __restrict__ p, float& ux, float& uy, float& uz) {
    const int4 q = s.pairs[c];
    const float4 b = s.bary[c];
    const float4 p0 = p[q.x], p1 = p[q.y], p2 = p[q.z], p3 = p[q.w];
    const float4 kc = s.kc[c];
    ux = b.x * p0.x + b.y * p1.x + b.z * p2.x + b.w * p3.x;
    uy = b.x * p0.y + b.y * p1.y + b.z * p2.y + b.w * p3.y;
    uz = b.x * p0.z + b.y * p1.z + b.z * p2.z + b.w * p3.z;
    ux = ux + kc.x;
    uy = uy + kc.y;
    uz = uz + kc.z;
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

// p_i += sum_c Gamma_c,i du_c over the incidence list of vertex i, entries
// [b, e) (update_p, contact_solver.cu:381-399).
ADMM_DEV void contact_gather_one(const DevScene& s, int i, int b, int e) {
    float dx = 0.f, dy = 0.f, dz = 0.f;
    for (int k = b; k < e; k++) {
        const int slot = s.vlist[k];
        const int c = slot >> 2;
        const float g = comp(s.gamma[c], slot & 3);
        const float4 d = s.du[c];
        dx = dx + d.x * g;
        dy = dy + d.y * g;
        dz = dz + d.z * g;
    }
    float4 p = s.p[i];
    p.x += dx;
    p.y += dy;
    p.z += dz;
    s.p[i] = p;
}

__global__ void __launch_bounds__(kContactThreads) k_contact_gather(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.nd) return;
    const int b = s.vstart[i], e = s.vstart[i + 1];
    if (b == e) return;
    contact_gather_one(s, i, b, e);
}

// One whole Jacobi pass of the contact solve in one kernel (k_contact_du and
// k_contact_gather fused): every vertex with contacts recomputes the du of its
// incident contacts from the previous pass's p (pin) and r (rin) -- the same
// arithmetic as k_contact_du -- and sums them in incidence-list order into
// pout; r_c + du_c goes to rout, written by the contact's lowest slot that holds
// a dynamic vertex.  Bit-identical to the two-kernel pass, half the launches.
__global__ void __launch_bounds__(kContactThreads) k_contact_pass(DevScene s, const float4* __restrict__ pin,
                                                                  float4* __restrict__ pout,
                                                                  const float4* __restrict__ rin,
                                                                  float4* __restrict__ rout) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.nd) return;
    const int b = s.vstart[i], e = s.vstart[i + 1];
    if (b == e) return;
    float dx = 0.f, dy = 0.f, dz = 0.f;
    for (int k = b; k < e; k++) {
        const int slot = s.vlist[k];
        const int c = slot >> 2;
        float ux, uy, uz;
        contact_u(s, c, pin, ux, uy, uz);
        const float4 r = rin[c];
        const float4 d = friction_cone_du(s, c, ux, uy, uz, r);
        const float g = comp(s.gamma[c], slot & 3);
        dx = dx + d.x * g;
        dy = dy + d.y * g;
        dz = dz + d.z * g;
        const int4 q = s.pairs[c];
        const int writer = q.x < s.nd ? 0 : q.y < s.nd ? 1 : q.z < s.nd ? 2 : 3;
        if ((slot & 3) == writer) rout[c] = f4(r.x + d.x, r.y + d.y, r.z + d.z);
    }
    float4 p = pin[i];
    p.x += dx;
    p.y += dy;
    p.z += dz;
    pout[i] = p;
}

// Copies p and r of the vertices / contacts that the passes update back from
// the second buffers (odd pass counts).
__global__ void __launch_bounds__(kContactThreads) k_contact_pass_copy(DevScene s, const float4* __restrict__ pin,
                                                                       const float4* __restrict__ rin) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s.nd && s.vstart[i] != s.vstart[i + 1]) s.p[i] = pin[i];
    const int nc = ccount(s);
    for (int c = i; c < nc; c += gridDim.x * blockDim.x) {
        const int4 q = s.pairs[c];
        if (q.x < s.nd || q.y < s.nd || q.z < s.nd || q.w < s.nd) s.rc[c] = rin[c];
    }
}

}  // namespace admm
