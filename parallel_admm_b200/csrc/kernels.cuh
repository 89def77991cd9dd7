// kernels.cuh -- per-iteration ADMM kernels (local step, dual updates, RHS,
// Jacobi sweeps, integration, residuals).
#pragma once
#include "contact.cuh"
#include "prox.cuh"
#include "scene_dev.cuh"

namespace admm {

constexpr int kLocalThreads = 128;
constexpr int kVertThreads = 128;

// ---------------------------------------------------------------------------
// Local step, fused with the elastic dual update of the previous iteration.
//   LOCAL_DUAL : Ue += D x - z            (admm_impl_gpu.cu:322-324)
//   LOCAL_PROX : z = prox(D x + Ue), y = z - Ue   (admm_impl_gpu.cu:52-59, 308)
// D x is evaluated from the vertex positions directly: F = E * Binv for
// triangles and tets (the rows of D are G = S * Binv, triangle_constraint.h:64-95,
// tetrahedral_constraint.h:58-89), the stored coefficients for bending and 1 for
// pins.  Blocks [0, tet_blocks) do tets, then triangles, bending, pins.
// ---------------------------------------------------------------------------
enum : int { LOCAL_PROX = 1, LOCAL_DUAL = 2 };

template <int MODE, int NR>
ADMM_DEV void finish_rows(const DevScene& s, int row, const float (&dx)[3 * NR], float (&zz)[3 * NR],
                          float4 (&ue)[NR]) {
#pragma unroll
    for (int r = 0; r < NR; r++) {
        ue[r] = s.ue[row + r];
        if (MODE & LOCAL_DUAL) {
            const float4 zo = s.z[row + r];
            ue[r].x = (dx[3 * r + 0] - zo.x) + ue[r].x;
            ue[r].y = (dx[3 * r + 1] - zo.y) + ue[r].y;
            ue[r].z = (dx[3 * r + 2] - zo.z) + ue[r].z;
            ue[r].w = 0.f;
        }
        zz[3 * r + 0] = dx[3 * r + 0] + ue[r].x;
        zz[3 * r + 1] = dx[3 * r + 1] + ue[r].y;
        zz[3 * r + 2] = dx[3 * r + 2] + ue[r].z;
    }
}

template <int MODE, int NR>
ADMM_DEV void store_rows(const DevScene& s, int row, const float (&zz)[3 * NR], const float4 (&ue)[NR]) {
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (MODE & LOCAL_DUAL) s.ue[row + r] = ue[r];
        if (MODE & LOCAL_PROX) {
            const float4 zr = f4(zz[3 * r], zz[3 * r + 1], zz[3 * r + 2]);
            s.z[row + r] = zr;
            s.y[row + r] = f4(zr.x - ue[r].x, zr.y - ue[r].y, zr.z - ue[r].z);
        }
    }
}

// D x rows of tet c from its (already loaded) indices and Binv rows.
ADMM_DEV void tet_dx_from(const float4* __restrict__ x, int4 id, float4 B0, float4 B1, float4 B2, float (&dx)[9]) {
    const float4 p0 = x[id.x], p1 = x[id.y], p2 = x[id.z], p3 = x[id.w];
    const float4 e0 = sub3(p1, p0), e1 = sub3(p2, p0), e2 = sub3(p3, p0);
    const float b[3][3] = {{B0.x, B0.y, B0.z}, {B1.x, B1.y, B1.z}, {B2.x, B2.y, B2.z}};
#pragma unroll
    for (int r = 0; r < 3; r++) {
        dx[3 * r + 0] = e0.x * b[0][r] + e1.x * b[1][r] + e2.x * b[2][r];
        dx[3 * r + 1] = e0.y * b[0][r] + e1.y * b[1][r] + e2.y * b[2][r];
        dx[3 * r + 2] = e0.z * b[0][r] + e1.z * b[1][r] + e2.z * b[2][r];
    }
}

ADMM_DEV void tri_dx_from(const float4* __restrict__ x, int4 id, float4 B, float (&dx)[6]) {
    const float4 p0 = x[id.x], p1 = x[id.y], p2 = x[id.z];
    const float4 e0 = sub3(p1, p0), e1 = sub3(p2, p0);
    dx[0] = e0.x * B.x + e1.x * B.z;
    dx[1] = e0.y * B.x + e1.y * B.z;
    dx[2] = e0.z * B.x + e1.z * B.z;
    dx[3] = e0.x * B.y + e1.x * B.w;
    dx[4] = e0.y * B.y + e1.y * B.w;
    dx[5] = e0.z * B.y + e1.z * B.w;
}

ADMM_DEV void tet_dx(const float4* __restrict__ x, const DevScene& s, int c, float (&dx)[9]) {
    const int4 id = s.tet_inds[c];
    const float4 p0 = x[id.x], p1 = x[id.y], p2 = x[id.z], p3 = x[id.w];
    const float4 e0 = sub3(p1, p0), e1 = sub3(p2, p0), e2 = sub3(p3, p0);
    const float4 B0 = s.tet_b0[c], B1 = s.tet_b1[c], B2 = s.tet_b2[c];
    const float b[3][3] = {{B0.x, B0.y, B0.z}, {B1.x, B1.y, B1.z}, {B2.x, B2.y, B2.z}};
#pragma unroll
    for (int r = 0; r < 3; r++) {
        dx[3 * r + 0] = e0.x * b[0][r] + e1.x * b[1][r] + e2.x * b[2][r];
        dx[3 * r + 1] = e0.y * b[0][r] + e1.y * b[1][r] + e2.y * b[2][r];
        dx[3 * r + 2] = e0.z * b[0][r] + e1.z * b[1][r] + e2.z * b[2][r];
    }
}

ADMM_DEV void tri_dx(const float4* __restrict__ x, const DevScene& s, int c, float (&dx)[6]) {
    const int4 id = s.tri_inds[c];
    const float4 p0 = x[id.x], p1 = x[id.y], p2 = x[id.z];
    const float4 e0 = sub3(p1, p0), e1 = sub3(p2, p0);
    const float4 B = s.tri_binv[c];  // B00 B01 B10 B11
    dx[0] = e0.x * B.x + e1.x * B.z;
    dx[1] = e0.y * B.x + e1.y * B.z;
    dx[2] = e0.z * B.x + e1.z * B.z;
    dx[3] = e0.x * B.y + e1.x * B.w;
    dx[4] = e0.y * B.y + e1.y * B.w;
    dx[5] = e0.z * B.y + e1.z * B.w;
}

ADMM_DEV void bend_dx(const float4* __restrict__ x, const DevScene& s, int c, float (&dx)[3]) {
    float ax = 0.f, ay = 0.f, az = 0.f;
    const int b = s.bend_off[c], e = s.bend_off[c + 1];
    for (int k = b; k < e; k++) {
        const float w = s.bend_coef[k];
        const float4 p = x[s.bend_inds[k]];
        ax += w * p.x;
        ay += w * p.y;
        az += w * p.z;
    }
    dx[0] = ax; dx[1] = ay; dx[2] = az;
}

template <int MODE>
__global__ void __launch_bounds__(kLocalThreads) k_local(DevScene s, int tet_blocks, int tri_blocks, int bend_blocks) {
    // constraint records are constant: they are loaded before the programmatic wait
    ADMM_PDL_TRIGGER();
    int blk = blockIdx.x;
    if (blk < tet_blocks) {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c >= s.ntet) return;
        const int4 id = __ldg(&s.tet_inds[c]);
        const float4 B0 = __ldg(&s.tet_b0[c]), B1 = __ldg(&s.tet_b1[c]), B2 = __ldg(&s.tet_b2[c]);
        ADMM_PDL_WAIT();
        float dx[9], zz[9];
        float4 ue[3];
        tet_dx_from(s.x, id, B0, B1, B2, dx);
        const int row = s.tet_sr + 3 * c;
        finish_rows<MODE, 3>(s, row, dx, zz, ue);
        if (MODE & LOCAL_PROX) prox_tet(zz);
        store_rows<MODE, 3>(s, row, zz, ue);
        return;
    }
    blk -= tet_blocks;
    if (blk < tri_blocks) {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c >= s.ntri) return;
        const int4 id = __ldg(&s.tri_inds[c]);
        const float4 Bt = __ldg(&s.tri_binv[c]);
        ADMM_PDL_WAIT();
        float dx[6], zz[6];
        float4 ue[2];
        tri_dx_from(s.x, id, Bt, dx);
        const int row = s.tri_sr + 2 * c;
        finish_rows<MODE, 2>(s, row, dx, zz, ue);
        if (MODE & LOCAL_PROX) prox_tri(zz);
        store_rows<MODE, 2>(s, row, zz, ue);
        return;
    }
    blk -= tri_blocks;
    if (blk < bend_blocks) {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c >= s.nbend) return;
        ADMM_PDL_WAIT();
        float dx[3], zz[3];
        float4 ue[1];
        bend_dx(s.x, s, c, dx);
        const int row = s.bend_sr + c;
        finish_rows<MODE, 1>(s, row, dx, zz, ue);
        if (MODE & LOCAL_PROX) prox_bend(zz, s.bend_rest[c]);
        store_rows<MODE, 1>(s, row, zz, ue);
        return;
    }
    blk -= bend_blocks;
    {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c >= s.npin) return;
        const int pi = __ldg(&s.pin_inds[c]);
        ADMM_PDL_WAIT();
        const float4 p = s.x[pi];
        float dx[3] = {p.x, p.y, p.z}, zz[3];
        float4 ue[1];
        const int row = s.pin_sr + c;
        finish_rows<MODE, 1>(s, row, dx, zz, ue);
        if (MODE & LOCAL_PROX) {
            const float4 q = s.pin_pos[c];
            zz[0] = q.x; zz[1] = q.y; zz[2] = q.z;
        }
        store_rows<MODE, 1>(s, row, zz, ue);
    }
}

// ---------------------------------------------------------------------------
// Pre-integration (do_integration_kernel, jacobi_solver.cu:183-215), plus the
// p <- v copy of the static range (admm_impl_gpu.cu:282).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kVertThreads) k_pre_integration(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    float4 x0 = s.x0[i], v = s.v[i], x;
    if (s.fixed[i] == 0) {
        if (i < s.nd) {
            v.y -= s.g * s.dt;
            x = f4(x0.x + v.x * s.dt, x0.y + v.y * s.dt, x0.z + v.z * s.dt);
        } else {
            x = f4(x0.x, x0.y, x0.z);
        }
    } else {
        v = f4(0.f, 0.f, 0.f);
        x = f4(x0.x, x0.y, x0.z);
    }
    const float m = s.mass[i];
    s.v[i] = v;
    s.x[i] = x;
    s.mxt[i] = f4(m * x.x, m * x.y, m * x.z);
    if (i >= s.nd) s.p[i] = v;
}

// ---------------------------------------------------------------------------
// Contact velocities, fused with the contact dual update of the previous
// iteration and the warm start of the contact projection:
//   DUALC : Uc += (x - x0) - h p           (admm_impl_gpu.cu:326-331)
//   p = ((x - x0) + Uc) / h                (admm_impl_gpu.cu:296-298)
//   WARM  : p += sum_c Gamma_c,i r_c        (update_p_kernel, contact_solver.cu:316-335)
// ---------------------------------------------------------------------------
// p = (x - x0 + Uc) / h (after Uc += (x - x0) - h p when DUALC), plus the warm
// start p += sum_c Gamma_c,i r_c over the incidence list of a vertex with
// contacts.  Blocks [0, split) take the dynamic vertices without contacts, one
// thread each; the others walk the touched list with kGatherLanes lanes per
// vertex.
template <bool DUALC>
ADMM_DEV float4 contact_p_base(const DevScene& s, int i) {
    const float4 x = s.x[i], x0 = s.x0[i];
    float4 uc = s.uc[i];
    if (DUALC) {
        const float4 p = s.p[i];
        uc.x = uc.x + ((x.x - x0.x) - p.x * s.dt);
        uc.y = uc.y + ((x.y - x0.y) - p.y * s.dt);
        uc.z = uc.z + ((x.z - x0.z) - p.z * s.dt);
        s.uc[i] = uc;
    }
    return f4(((x.x - x0.x) + uc.x) * s.dt_inv, ((x.y - x0.y) + uc.y) * s.dt_inv, ((x.z - x0.z) + uc.z) * s.dt_inv);
}

// Waits before it triggers (so does every kernel of the projection passes after
// it): each pass may load the detection's contact data before its own wait.
template <bool DUALC>
__global__ void __launch_bounds__(kVertThreads) k_contact_p(DevScene s, int split) {
    ADMM_PDL_WAIT_THEN_TRIGGER();
    if ((int)blockIdx.x < split) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i < s.nd && s.vstart[i] == s.vstart[i + 1]) s.p[i] = contact_p_base<DUALC>(s, i);
        return;
    }
    const int sub = threadIdx.x % kGatherLanes;
    const unsigned gmask = 0xffu << (threadIdx.x & 31 & ~(kGatherLanes - 1));
    const int ntv = *s.ntv;
    const int g0 = ((blockIdx.x - split) * blockDim.x + threadIdx.x) / kGatherLanes;
    const int gs = (gridDim.x - split) * blockDim.x / kGatherLanes;
    for (int t = g0; t < ntv; t += gs) {
        const int4 r = s.tvr[t];  // the vertex and its list bounds in one load
        const int i = r.x;
        if (i >= s.nd) continue;
        const float4 warm = gather_group(s, s.rc, r.y, r.z, sub, gmask);
        if (sub == 0) {
            float4 p = contact_p_base<DUALC>(s, i);
            p.x += warm.x;
            p.y += warm.y;
            p.z += warm.z;
            s.p[i] = p;
        }
    }
}

// Gather of one sliced-ELL row: the warp `w` (a slice) accumulates sum val * v[col]
// for its 32/T rows; lanes of one row are reduced with shuffles.  Returns the
// row's sum in every lane of the row; `row` receives the lane's row index.
// CG = true reads v through L2 only (ld.global.cg): v is written by other
// blocks of a persistent kernel while this one runs.
template <int T, bool CG = false>
ADMM_DEV float4 ell_row_sum(const SlicedEll& M, const float4* __restrict__ v, int w, int lane, int& row) {
    constexpr int S = 32 / T;
    row = M.rowid ? __ldg(&M.rowid[w * S + (lane % S)]) : w * S + (lane % S);
    const int b = M.ptr[w], e = M.ptr[w + 1];
    float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll 4
    for (int k = b + lane; k < e; k += 32) {
        const int c = __ldg(&M.col[k]);
        const float a = __ldg(&M.val[k]);
        const float4 q = CG ? __ldcg(&v[c]) : v[c];
        ax = fmaf(a, q.x, ax);
        ay = fmaf(a, q.y, ay);
        az = fmaf(a, q.z, az);
    }
#pragma unroll
    for (int o = S; o < 32; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    return f4(ax, ay, az);
}

// ---------------------------------------------------------------------------
// Right-hand side (admm_impl_gpu.cu:307-318):
//   b = M x~ + h^2 D^T W^2 (z - Ue) [+ h^2 W_c (h p + x0 - Uc)]
// as a gather over the sliced-ELL copy of h^2 D^T W^2 (one warp per slice).
// SAVE_PREV also keeps x before the solve (for the dual residual).
// ---------------------------------------------------------------------------
// b_i from the row sum acc = (h^2 D^T W^2 (z - Ue))_i.
ADMM_DEV float4 rhs_value(const DevScene& s, float4 acc, float4 m, float4 p, float4 x0, float4 uc, float wc) {
    float4 bi = f4(m.x + acc.x, m.y + acc.y, m.z + acc.z);
    if (s.contact) {
        bi.x = bi.x + wc * ((p.x * s.dt + x0.x) - uc.x);
        bi.y = bi.y + wc * ((p.y * s.dt + x0.y) - uc.y);
        bi.z = bi.z + wc * ((p.z * s.dt + x0.z) - uc.z);
    }
    return bi;
}

template <bool SAVE_PREV>
ADMM_DEV void rhs_row(const DevScene& s, int i, float4 acc) {
    const float4 z = f4(0.f, 0.f, 0.f);
    const bool c = s.contact;
    s.b[i] = rhs_value(s, acc, s.mxt[i], c ? s.p[i] : z, c ? s.x0[i] : z, c ? s.uc[i] : z, c ? s.dt2wc[i] : 0.f);
    if (SAVE_PREV) s.xprev[i] = s.x[i];
}

// ell_row_sum in two parts around the programmatic-dependency wait: load()
// reads the lane's row index and the matrix entries of its first kPrefetch
// steps (the matrix is constant, so before the wait), sum() the gathered vector
// and the rest of the row (after it).  Between the two a kernel loads its own
// per-row operands, so that they travel in parallel with the gathers instead of
// after the row sum.  Same operations in the same order as ell_row_sum.
constexpr int kPrefetch = 8;

// LONG: rows much longer than kPrefetch * 32 / (32 / T) entries (R, whose rows
// hold every constraint row of a vertex): the rest of the row is unrolled so
// that several of its loads are in flight; the sweep's short rows (A) keep the
// plain loop, which measured faster there.
template <int T, bool LONG = false>
struct EllRowPf {
    static constexpr int S = 32 / T;
    int row, b, e;
    int cc[kPrefetch];
    float vv[kPrefetch];

    ADMM_DEV void load(const SlicedEll& M, int w, int lane) {
        row = M.rowid ? __ldg(&M.rowid[w * S + (lane % S)]) : w * S + (lane % S);
        b = M.ptr[w];
        e = M.ptr[w + 1];
#pragma unroll
        for (int j = 0; j < kPrefetch; j++) {
            const int k = b + lane + 32 * j;
            cc[j] = k < e ? __ldg(&M.col[k]) : 0;
            vv[j] = k < e ? __ldg(&M.val[k]) : 0.f;
        }
    }

    ADMM_DEV float4 sum(const SlicedEll& M, const float4* __restrict__ v, int lane) const {
        float ax = 0.f, ay = 0.f, az = 0.f;
#pragma unroll
        for (int j = 0; j < kPrefetch; j++) {
            if (b + lane + 32 * j < e) {
                const float4 q = v[cc[j]];
                ax = fmaf(vv[j], q.x, ax);
                ay = fmaf(vv[j], q.y, ay);
                az = fmaf(vv[j], q.z, az);
            }
        }
        if (LONG) {
#pragma unroll 4
            for (int k = b + lane + 32 * kPrefetch; k < e; k += 32) {
                const int c = __ldg(&M.col[k]);
                const float a = __ldg(&M.val[k]);
                const float4 q = v[c];
                ax = fmaf(a, q.x, ax);
                ay = fmaf(a, q.y, ay);
                az = fmaf(a, q.z, az);
            }
        } else {
            for (int k = b + lane + 32 * kPrefetch; k < e; k += 32) {
                const int c = __ldg(&M.col[k]);
                const float a = __ldg(&M.val[k]);
                const float4 q = v[c];
                ax = fmaf(a, q.x, ax);
                ay = fmaf(a, q.y, ay);
                az = fmaf(a, q.z, az);
            }
        }
#pragma unroll
        for (int o = S; o < 32; o <<= 1) {
            ax += __shfl_xor_sync(0xffffffffu, ax, o);
            ay += __shfl_xor_sync(0xffffffffu, ay, o);
            az += __shfl_xor_sync(0xffffffffu, az, o);
        }
        return f4(ax, ay, az);
    }
};

template <int T, bool SAVE_PREV>
__global__ void __launch_bounds__(kVertThreads) k_rhs(DevScene s) {
    ADMM_PDL_TRIGGER();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= s.R.nslices) return;
    EllRowPf<T, true> r;
    r.load(s.R, w, lane);
    const int i = r.row;
    const bool own = i < s.nd, c = own && s.contact;
    const float wc = c ? __ldg(&s.dt2wc[i]) : 0.f;
    ADMM_PDL_WAIT();
    const float4 z = f4(0.f, 0.f, 0.f);
    const float4 m = own ? s.mxt[i] : z, p = c ? s.p[i] : z, x0 = c ? s.x0[i] : z, uc = c ? s.uc[i] : z;
    const float4 xi = SAVE_PREV && own ? s.x[i] : z;
    const float4 acc = r.sum(s.R, s.y, lane);
    if (lane >= 32 / T || !own) return;
    s.b[i] = rhs_value(s, acc, m, p, x0, uc, wc);
    if (SAVE_PREV) s.xprev[i] = xi;
}

// dst_i = (b_i - acc) / a_ii
ADMM_DEV void jacobi_row(const DevScene& s, int i, float4 acc, float4* __restrict__ dst) {
    const float4 bi = s.b[i];
    const float d = s.a_diag[i];
    dst[i] = f4((bi.x - acc.x) / d, (bi.y - acc.y) / d, (bi.z - acc.z) / d);
}

// ---------------------------------------------------------------------------
// One Jacobi sweep (JacobiFunctor, jacobi_solver.cu:52-98):
//   dst_i = (b_i - sum_{j != i} a_ij src_j) / a_ii
// over the sliced-ELL copy of the off-diagonal part of A (one warp per slice).
// ---------------------------------------------------------------------------
// Capped at 32 registers (16 blocks of 128 threads per SM, all 64 warps resident): the sweep
// waits on its gathers, and the extra resident warps hide more of that latency than the
// 8 bytes of spill cost (batch: 52.9 -> 49.5 us per sweep in the step graph).
template <int T>
__global__ void __launch_bounds__(kVertThreads, 16) k_jacobi(DevScene s, const float4* __restrict__ src,
                                                             float4* __restrict__ dst) {
    ADMM_PDL_TRIGGER();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= s.A.nslices) return;
    EllRowPf<T> r;
    r.load(s.A, w, lane);
    const int i = r.row;
    const bool own = i < s.nd;
    const float d = own ? __ldg(&s.a_diag[i]) : 1.f;  // A is constant: before the wait
    ADMM_PDL_WAIT();
    const float4 bi = own ? s.b[i] : f4(0.f, 0.f, 0.f);
    const float4 acc = r.sum(s.A, src, lane);
    if (lane >= 32 / T || !own) return;
    dst[i] = f4((bi.x - acc.x) / d, (bi.y - acc.y) / d, (bi.z - acc.z) / d);
}

// ---------------------------------------------------------------------------
// Two Jacobi sweeps in one launch (jacobi_mode 3).  One block per row tile:
// phase 1 computes the first sweep for the tile's own and halo rows from the
// global src into shared memory, phase 2 the second sweep for the own rows
// from shared memory into dst.  Every row is summed with the same entries in
// the same order and lane layout as k_jacobi, so two launches of k_jacobi and
// one of k_jacobi2 give identical bits; the halo rows are computed twice (by
// their own tile and by their neighbours'), the price of half the launches.
// ---------------------------------------------------------------------------
constexpr int kTileThreads = 1024;
constexpr int kTileOwn = 64;

template <int T>
__global__ void __launch_bounds__(kTileThreads) k_jacobi2(DevScene s, TileSet ts, const float4* __restrict__ src,
                                                          float4* __restrict__ dst) {
    ADMM_PDL_PROLOGUE();
    extern __shared__ float4 ysh[];
    constexpr int S = 32 / T;
    const int t = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int r0 = ts.row0[t], n1 = ts.nlocal[t], no = ts.nown[t];
    const int a1 = ts.s1_0[t], b1 = a1 + ts.s1_n[t];
    for (int w = a1 + warp; w < b1; w += nw) {
        int lr;
        const float4 acc = ell_row_sum<T>(ts.e1, src, w, lane, lr);
        const int li = lr - a1 * S;
        if (lane < S && li < n1) {
            const int g = ts.trow[r0 + li];
            const float4 bi = s.b[g];
            const float d = s.a_diag[g];
            ysh[li] = f4((bi.x - acc.x) / d, (bi.y - acc.y) / d, (bi.z - acc.z) / d);
        }
    }
    __syncthreads();
    const int a2 = ts.s2_0[t], b2 = a2 + ts.s2_n[t];
    for (int w = a2 + warp; w < b2; w += nw) {
        int lr;
        const float4 acc = ell_row_sum<T>(ts.e2, ysh, w, lane, lr);
        const int li = lr - a2 * S;
        if (lane < S && li < no) jacobi_row(s, ts.trow[r0 + li], acc, dst);
    }
}

// ---------------------------------------------------------------------------
// The whole global step in one persistent kernel: the right-hand side (RHS)
// and `sweeps` Jacobi sweeps, bit-identical to k_rhs + k_jacobi launches.
//
// Block g owns rows [g*RB, (g+1)*RB) (RB a multiple of 32, so that the slices
// of both sliced-ELL matrices align with the blocks).  After every sweep a
// block publishes the number of sweeps it has completed in epoch[g]
// (st.release.gpu after a block barrier); before sweep k it waits until every
// block in its dependency list -- the owners of the columns of its rows,
// symmetrised -- has completed sweep k-1 (ld.acquire.gpu).  That one wait
// covers both hazards of the ping-pong buffers: the values it reads are
// complete, and no neighbour still reads the buffer it is about to overwrite.
// Epoch counters only grow (wrap-safe comparisons); all blocks hold the same
// count between launches, so each launch takes its own block's count as base.
// Every wait is bounded by spin_limit polls; on expiry the block sets err[3]
// and returns, and the blocks waiting on it expire in turn.  All blocks must
// be co-resident: the launch is cooperative.
// ---------------------------------------------------------------------------
constexpr int kPersistThreads = 512;

ADMM_DEV unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
ADMM_DEV void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <int T, int TR, bool RHS, bool SAVE_PREV>
__global__ void __launch_bounds__(kPersistThreads, 1) k_global_persist(DevScene s, PersistPlan pp, int sweeps) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __shared__ unsigned sh_base;
    __shared__ int sh_abort;
    const int g = blockIdx.x;
    const int r0 = g * pp.rows_per_block, r1 = min(s.nd, r0 + pp.rows_per_block);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        sh_base = ld_acquire_u32(pp.epoch + g);
        sh_abort = 0;
    }
    if (RHS) {
        constexpr int SR = 32 / TR;
        const int w1 = (r1 + SR - 1) / SR;
        for (int w = r0 / SR + warp; w < w1; w += nw) {
            int i;
            const float4 acc = ell_row_sum<TR>(s.R, s.y, w, lane, i);
            if (lane < SR && i < r1) rhs_row<SAVE_PREV>(s, i, acc);
        }
    }
    __syncthreads();
    const unsigned base = sh_base;
    constexpr int S = 32 / T;
    const int w1 = (r1 + S - 1) / S;
    const int d0 = pp.dep_ptr[g], d1 = pp.dep_ptr[g + 1];
    for (int k = 0; k < sweeps; k++) {
        if (k > 0) {
            if (warp == 0) {
                const unsigned target = base + (unsigned)k;
                bool ok = true;
                for (int d = d0 + lane; d < d1 && ok; d += 32) {
                    const unsigned* e = pp.epoch + pp.dep_idx[d];
                    int spins = 0;
                    while ((int)(ld_acquire_u32(e) - target) < 0) {
                        if (++spins > pp.spin_limit) {
                            ok = false;
                            break;
                        }
                        if (spins > 32) __nanosleep(64);
                    }
                }
                if (__any_sync(0xffffffffu, !ok) && lane == 0) {
                    sh_abort = 1;
                    s.err[3] = 1;
                }
            }
            __syncthreads();
            if (sh_abort) return;
        }
        const float4* src = k == 0 ? s.x : s.jac[(k - 1) & 1];
        float4* dst = k == sweeps - 1 ? s.x : s.jac[k & 1];
        for (int w = r0 / S + warp; w < w1; w += nw) {
            int i;
            const float4 acc = ell_row_sum<T, true>(s.A, src, w, lane, i);
            if (lane < S && i < r1) jacobi_row(s, i, acc, dst);
        }
        __syncthreads();
        if (threadIdx.x == 0) st_release_u32(pp.epoch + g, base + (unsigned)k + 1u);
    }
}

// ---------------------------------------------------------------------------
// Preconditioned conjugate gradients for the global step (global_solver > 0),
// an addition with no counterpart in the reference.  A (x) I3 is
// solved for the three coordinate columns at once (one 3nd-vector CG, so that
// a 3x3 block preconditioner may couple them), warm-started from the current x.
// Chronopoulos-Gear form: one reduction pair per iteration, two kernels:
//   KA (k_pcg_update): alpha, beta from the reduced (gamma, delta);
//        p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s, u = M^-1 r
//   KB (k_pcg_spmv):   w = A u, per-block partial sums of (r, u) and (w, u)
// Reductions are deterministic: each block writes its FP64 partials, every
// block of the next kernel sums all of them in the same order.  The scalars
// (gamma, alpha) of iteration i live in scal[i & 1].
// ---------------------------------------------------------------------------
struct PcgDev {
    float4 *r = nullptr, *u = nullptr, *w = nullptr, *p = nullptr, *s = nullptr;
    double* part = nullptr;        // [2 * blocks] gamma partials, then delta partials
    double* scal = nullptr;        // [2 x 4] per iteration parity: gamma, alpha
    const float* block = nullptr;  // [9 * nd] per-vertex 3x3 preconditioner blocks (row-major), or null
    int blocks = 0;                // grid of k_pcg_spmv (= number of partials)
};

ADMM_DEV float4 pcg_precond(const DevScene& s, const PcgDev& g, int i, float4 r) {
    if (g.block) {
        const float* B = g.block + 9 * (size_t)i;
        return f4(B[0] * r.x + B[1] * r.y + B[2] * r.z, B[3] * r.x + B[4] * r.y + B[5] * r.z,
                  B[6] * r.x + B[7] * r.y + B[8] * r.z);
    }
    const float d = s.a_diag[i];
    return f4(r.x / d, r.y / d, r.z / d);
}

ADMM_DEV double dot3d(float4 a, float4 b) {
    return (double)a.x * (double)b.x + (double)a.y * (double)b.y + (double)a.z * (double)b.z;
}

// Sum of the n partials at part (every block, same order); result in all threads.
ADMM_DEV double pcg_reduce(const double* __restrict__ part, int n, double* sh) {
    double v = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) v += part[k];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) sh[32] = v;
    __syncthreads();
    const double r = sh[32];
    __syncthreads();
    return r;
}

// w = A v for the rows of slice w (lanes of a row hold the result), A = diag + off-diagonal ELL.
template <int T>
ADMM_DEV float4 pcg_apply(const DevScene& s, const float4* __restrict__ v, int wslice, int lane, int& row) {
    const float4 acc = ell_row_sum<T>(s.A, v, wslice, lane, row);
    if (row >= s.nd) return acc;
    const float d = s.a_diag[row];
    const float4 vi = v[row];
    return f4(fmaf(d, vi.x, acc.x), fmaf(d, vi.y, acc.y), fmaf(d, vi.z, acc.z));
}

// Init, part 1: r = b - A x, u = M^-1 r, p = s = 0 (with beta = 0 the first update sets p = u, s = w).
template <int T>
__global__ void __launch_bounds__(kVertThreads) k_pcg_init(DevScene s, PcgDev g) {
    ADMM_PDL_PROLOGUE();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= s.A.nslices) return;
    int i;
    const float4 ax = pcg_apply<T>(s, s.x, w, lane, i);
    if (lane >= 32 / T || i >= s.nd) return;
    const float4 b = s.b[i];
    const float4 r = f4(b.x - ax.x, b.y - ax.y, b.z - ax.z);
    g.r[i] = r;
    g.u[i] = pcg_precond(s, g, i, r);
    g.p[i] = f4(0.f, 0.f, 0.f);
    g.s[i] = f4(0.f, 0.f, 0.f);
}

// KB: w = A u and the block partials of (r, u), (w, u).
template <int T>
__global__ void __launch_bounds__(kVertThreads) k_pcg_spmv(DevScene s, PcgDev g) {
    ADMM_PDL_PROLOGUE();
    __shared__ double sh[40];
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double ga = 0.0, de = 0.0;
    if (w < s.A.nslices) {
        int i;
        const float4 au = pcg_apply<T>(s, g.u, w, lane, i);
        if (lane < 32 / T && i < s.nd) {
            g.w[i] = au;
            const float4 u = g.u[i];
            ga = dot3d(g.r[i], u);
            de = dot3d(au, u);
        }
    }
    ga = block_sum(ga, sh);
    de = block_sum(de, sh);
    if (threadIdx.x == 0) {
        g.part[blockIdx.x] = ga;
        g.part[g.blocks + blockIdx.x] = de;
    }
}

// KA of iteration `it` (it = 0: beta = 0, alpha = gamma / delta).
__global__ void __launch_bounds__(kVertThreads) k_pcg_update(DevScene s, PcgDev g, int it) {
    ADMM_PDL_PROLOGUE();
    __shared__ double sh[40];
    const double gamma = pcg_reduce(g.part, g.blocks, sh);
    const double delta = pcg_reduce(g.part + g.blocks, g.blocks, sh);
    double alpha, beta;
    if (it == 0) {
        beta = 0.0;
        alpha = delta != 0.0 ? gamma / delta : 0.0;
    } else {
        const double* prev = g.scal + 4 * ((it - 1) & 1);
        beta = prev[0] != 0.0 ? gamma / prev[0] : 0.0;
        const double den = delta - beta * gamma / (prev[1] != 0.0 ? prev[1] : 1.0);
        alpha = den != 0.0 ? gamma / den : 0.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double* cur = g.scal + 4 * (it & 1);
        cur[0] = gamma;
        cur[1] = alpha;
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.nd) return;
    const float a = (float)alpha, bt = (float)beta;
    const float4 u = g.u[i], w = g.w[i];
    float4 p = g.p[i], sv = g.s[i], x = s.x[i], r = g.r[i];
    p = f4(fmaf(bt, p.x, u.x), fmaf(bt, p.y, u.y), fmaf(bt, p.z, u.z));
    sv = f4(fmaf(bt, sv.x, w.x), fmaf(bt, sv.y, w.y), fmaf(bt, sv.z, w.z));
    x = f4(fmaf(a, p.x, x.x), fmaf(a, p.y, x.y), fmaf(a, p.z, x.z));
    r = f4(fmaf(-a, sv.x, r.x), fmaf(-a, sv.y, r.y), fmaf(-a, sv.z, r.z));
    g.p[i] = p;
    g.s[i] = sv;
    s.x[i] = x;
    g.r[i] = r;
    g.u[i] = pcg_precond(s, g, i, r);
}

// The CPU backend's b_ini = Damp x0 (admm_impl_cpu.cpp:295), added to every
// right-hand side (:344): folded into M x~, which every right-hand side starts from.
__global__ void __launch_bounds__(kVertThreads) k_damp_binit(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.nd) return;
    const float4 xi = s.x0[i];
    const float d = s.dmp_diag[i];
    float ax = d * xi.x, ay = d * xi.y, az = d * xi.z;
    for (int k = s.dmp_start[i]; k < s.dmp_start[i + 1]; k++) {
        const float4 xj = s.x0[s.dmp_col[k]];
        const float a = s.dmp_val[k];
        ax = fmaf(a, xj.x, ax);
        ay = fmaf(a, xj.y, ay);
        az = fmaf(a, xj.z, az);
    }
    float4 m = s.mxt[i];
    m.x += ax;
    m.y += ay;
    m.z += az;
    s.mxt[i] = m;
}

__global__ void k_copy_dyn(DevScene s, const float4* __restrict__ src, float4* __restrict__ dst) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < s.nd) dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// End of step: the last contact dual update, then do_post_process_kernel
// (jacobi_solver.cu:236-252): v = (x - x0)/h on dynamic vertices, x0 = x.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kVertThreads) k_vertex_final(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    const float4 x = s.x[i], x0 = s.x0[i];
    if (i < s.nd) {
        if (s.contact) {
            const float4 p = s.p[i];
            float4 uc = s.uc[i];
            uc.x = uc.x + ((x.x - x0.x) - p.x * s.dt);
            uc.y = uc.y + ((x.y - x0.y) - p.y * s.dt);
            uc.z = uc.z + ((x.z - x0.z) - p.z * s.dt);
            s.uc[i] = uc;
        }
        s.v[i] = f4((x.x - x0.x) * s.dt_inv, (x.y - x0.y) * s.dt_inv, (x.z - x0.z) * s.dt_inv);
    }
    s.x0[i] = f4(x.x, x.y, x.z);
}

// ---------------------------------------------------------------------------
// Residuals, FP64, after the global solve of an iteration (before its dual
// update).  With r_e = D x - z, r_c = x - x0 - h p (contact surface only):
//   primal^2 = sum w^2 |D x - z|^2 + sum w_c |x - x0 - h p|^2
//   dual^2   = sum w^2 |D (x - x_prev)|^2 + sum w_c |x - x_prev|^2
//   scale^2  = sum w^2 |z|^2 + sum w_c |x - x0|^2
// Accumulated into s.res[0..2] (zeroed by the caller).
// ---------------------------------------------------------------------------
template <int NR>
ADMM_DEV void res_rows(const DevScene& s, int row, const float (&dx)[3 * NR], const float (&dp)[3 * NR],
                       double& pr, double& du, double& sc) {
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const double w = s.wrow[row + r];
        const double w2 = w * w;
        const float4 z = s.z[row + r];
        const double e0 = (double)dx[3 * r] - z.x, e1 = (double)dx[3 * r + 1] - z.y, e2 = (double)dx[3 * r + 2] - z.z;
        const double d0 = (double)dx[3 * r] - dp[3 * r], d1 = (double)dx[3 * r + 1] - dp[3 * r + 1],
                     d2 = (double)dx[3 * r + 2] - dp[3 * r + 2];
        pr += w2 * (e0 * e0 + e1 * e1 + e2 * e2);
        du += w2 * (d0 * d0 + d1 * d1 + d2 * d2);
        sc += w2 * ((double)z.x * z.x + (double)z.y * z.y + (double)z.z * z.z);
    }
}

__global__ void __launch_bounds__(kLocalThreads) k_residual(DevScene s, int tet_blocks, int tri_blocks,
                                                           int bend_blocks, int pin_blocks) {
    ADMM_PDL_PROLOGUE();
    __shared__ double sh[kLocalThreads / 32];
    double pr = 0.0, du = 0.0, sc = 0.0;
    int blk = blockIdx.x;
    const float4* xp = s.xprev;
    if (blk < tet_blocks) {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c < s.ntet) {
            float dx[9], dp[9];
            tet_dx(s.x, s, c, dx);
            tet_dx(xp, s, c, dp);
            res_rows<3>(s, s.tet_sr + 3 * c, dx, dp, pr, du, sc);
        }
    } else if ((blk -= tet_blocks) < tri_blocks) {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c < s.ntri) {
            float dx[6], dp[6];
            tri_dx(s.x, s, c, dx);
            tri_dx(xp, s, c, dp);
            res_rows<2>(s, s.tri_sr + 2 * c, dx, dp, pr, du, sc);
        }
    } else if ((blk -= tri_blocks) < bend_blocks) {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c < s.nbend) {
            float dx[3], dp[3];
            bend_dx(s.x, s, c, dx);
            bend_dx(xp, s, c, dp);
            res_rows<1>(s, s.bend_sr + c, dx, dp, pr, du, sc);
        }
    } else if ((blk -= bend_blocks) < pin_blocks) {
        const int c = blk * kLocalThreads + threadIdx.x;
        if (c < s.npin) {
            const float4 a = s.x[s.pin_inds[c]], bp = xp[s.pin_inds[c]];
            float dx[3] = {a.x, a.y, a.z}, dp[3] = {bp.x, bp.y, bp.z};
            res_rows<1>(s, s.pin_sr + c, dx, dp, pr, du, sc);
        }
    } else {
        blk -= pin_blocks;
        const int i = blk * kLocalThreads + threadIdx.x;
        if (s.contact && i < s.nd && s.dt2wc[i] > 0.f) {
            const double w = s.cw[i];
            const float4 x = s.x[i], x0 = s.x0[i], p = s.p[i], q = xp[i];
            const double r0 = ((double)x.x - x0.x) - (double)s.dt * p.x;
            const double r1 = ((double)x.y - x0.y) - (double)s.dt * p.y;
            const double r2 = ((double)x.z - x0.z) - (double)s.dt * p.z;
            const double d0 = (double)x.x - q.x, d1 = (double)x.y - q.y, d2 = (double)x.z - q.z;
            const double s0 = (double)x.x - x0.x, s1 = (double)x.y - x0.y, s2 = (double)x.z - x0.z;
            pr += w * (r0 * r0 + r1 * r1 + r2 * r2);
            du += w * (d0 * d0 + d1 * d1 + d2 * d2);
            sc += w * (s0 * s0 + s1 * s1 + s2 * s2);
        }
    }
    pr = block_sum(pr, sh);
    du = block_sum(du, sh);
    sc = block_sum(sc, sh);
    if (threadIdx.x == 0) {  // per-block partials, summed in a fixed order by k_residual_reduce
        s.res_part[3 * blockIdx.x] = pr;
        s.res_part[3 * blockIdx.x + 1] = du;
        s.res_part[3 * blockIdx.x + 2] = sc;
    }
}

// res[0..2] = the sums of the n block partials of k_residual, in a fixed order
// (run to run identical residuals, hence identical convergence decisions).
__global__ void __launch_bounds__(256) k_residual_reduce(DevScene s, int n) {
    ADMM_PDL_PROLOGUE();
    __shared__ double sh[8];
    double v[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < n; b += blockDim.x)
        for (int k = 0; k < 3; k++) v[k] += s.res_part[3 * b + k];
    for (int k = 0; k < 3; k++) {
        const double t = block_sum(v[k], sh);
        if (threadIdx.x == 0) s.res[k] = t;
    }
}

// ---------------------------------------------------------------------------
// Convergence test after a chunk of ADMM iterations (residual_tol > 0): counts
// the chunk's iterations into iters[0] and keeps the WHILE node of the substep
// graph looping while the relative primal or dual residual is above `tol` and
// another chunk still fits in `max_iter` iterations.  One thread.
// ---------------------------------------------------------------------------
// The decision is also stored in done[1] (1 = another chunk), which the eager
// (profiling) path reads on the host; in_graph = 0 skips the graph condition.
__global__ void k_check_converged(DevScene s, cudaGraphConditionalHandle cond, float tol, int chunk, int max_iter,
                                  int in_graph) {
    ADMM_PDL_PROLOGUE();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int iters = s.done[0] + chunk;
    s.done[0] = iters;
    const double sc = s.res[2] > 0.0 ? sqrt(s.res[2]) : 1.0;
    const double pr = sqrt(s.res[0]) / sc, du = sqrt(s.res[1]) / sc;
    const bool more = (pr > (double)tol || du > (double)tol) && iters + chunk <= max_iter;
    s.done[1] = more ? 1 : 0;
    if (in_graph) cudaGraphSetConditional(cond, more ? 1u : 0u);
}

}  // namespace admm
