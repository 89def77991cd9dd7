// lbvh.cuh -- linear BVH over the surface triangles and surface edges, and the
// discrete collision detection (DCD) that runs on it.
//
// Build (per tree, every DCD): element boxes + scene box (one pass, ordered-int
// atomics), 63-bit Morton codes (21 bits per axis) of the box centres,
// stable radix sort, Karras' radix-tree construction (T. Karras, "Maximizing
// Parallelism in the Construction of BVHs, Octrees, and k-d Trees", HPG 2012)
// with the leaf index as tie-break for equal codes, and the atomic bottom-up
// refit.  The reference does the same steps with 30-bit codes and thrust
// (lbvh.cu:944-1034, 1468-1540).
//
// Traversal: one thread per query, a bounded stack, boxes tested with the
// reference's overlap rule (lbvh.cu:43-49) and the region-0 narrow phase of
// dist_g.cuh:29-513 evaluated with non-contracting float operations.  Pairs are
// emitted deterministically in two passes (count, scan, write), so the contact
// list is ordered by query and tree order, not by atomic arrival as in the
// reference (lbvh.cu:1644, 1672).
#pragma once
#include "common.cuh"
#include "scan_sort.cuh"
#include "scene_dev.cuh"

namespace admm {

// --------------------------- element boxes ---------------------------------
ADMM_DEV void box_add(float4& lo, float4& up, float4 p) {
    lo.x = fminf(lo.x, p.x); lo.y = fminf(lo.y, p.y); lo.z = fminf(lo.z, p.z);
    up.x = fmaxf(up.x, p.x); up.y = fmaxf(up.y, p.y); up.z = fmaxf(up.z, p.z);
}

template <int NV>
__global__ void __launch_bounds__(256) k_elem_boxes(const float4* __restrict__ x, const int* __restrict__ elems,
                                                   int elem_stride, int n, BvhDev t) {
    ADMM_PDL_PROLOGUE();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    float4 lo = f4(1e32f, 1e32f, 1e32f), up = f4(-1e32f, -1e32f, -1e32f);
    if (e < n) {
#pragma unroll
        for (int k = 0; k < NV; k++) box_add(lo, up, x[elems[e * elem_stride + k]]);
        t.elem_lo[e] = lo;
        t.elem_up[e] = up;
    }
    // scene box: warp reduce, one atomic per warp and component
    float v[6] = {lo.x, lo.y, lo.z, -up.x, -up.y, -up.z};
#pragma unroll
    for (int c = 0; c < 6; c++) {
        float a = v[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
        v[c] = a;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&t.scene[0], float_to_ordered(v[0]));
        atomicMin(&t.scene[1], float_to_ordered(v[1]));
        atomicMin(&t.scene[2], float_to_ordered(v[2]));
        atomicMax(&t.scene[3], float_to_ordered(-v[3]));
        atomicMax(&t.scene[4], float_to_ordered(-v[4]));
        atomicMax(&t.scene[5], float_to_ordered(-v[5]));
    }
}

__global__ void k_scene_init(BvhDev a, BvhDev b) {
    ADMM_PDL_PROLOGUE();
    const int i = threadIdx.x;
    if (i < 3) {
        a.scene[i] = float_to_ordered(3e38f);
        b.scene[i] = float_to_ordered(3e38f);
    } else if (i < 6) {
        a.scene[i] = float_to_ordered(-3e38f);
        b.scene[i] = float_to_ordered(-3e38f);
    }
}

// --------------------------- Morton codes ----------------------------------
ADMM_DEV unsigned long long spread21(unsigned int v) {
    unsigned long long x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__global__ void __launch_bounds__(256) k_morton(BvhDev t) {
    ADMM_PDL_PROLOGUE();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= t.n) return;
    const float slo[3] = {ordered_to_float(t.scene[0]), ordered_to_float(t.scene[1]), ordered_to_float(t.scene[2])};
    const float sup[3] = {ordered_to_float(t.scene[3]), ordered_to_float(t.scene[4]), ordered_to_float(t.scene[5])};
    const float4 lo = t.elem_lo[e], up = t.elem_up[e];
    const float c[3] = {(lo.x + up.x) * 0.5f, (lo.y + up.y) * 0.5f, (lo.z + up.z) * 0.5f};
    unsigned int q[3];
    const float res = 2097152.0f;  // 2^21
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float ext = sup[a] - slo[a];
        float u = ext > 0.f ? (c[a] - slo[a]) / ext : 0.5f;
        u = fminf(fmaxf(u * res, 0.f), res - 1.f);
        q[a] = (unsigned int)u;
    }
    t.keys[e] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    t.vals[e] = e;
}

// --------------------------- Karras build -----------------------------------
ADMM_DEV int karras_delta(const unsigned long long* __restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long a = k[i], b = k[j];
    if (a == b) return 64 + __clz((unsigned)(i ^ j));
    return __clzll((long long)(a ^ b));
}

// Internal node i in [0, n-1); leaf k is node n-1+k.  Also writes the sorted
// leaf records (element id and box) and clears the refit counters.
__global__ void __launch_bounds__(256) k_karras(BvhDev t) {
    ADMM_PDL_PROLOGUE();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = t.n;
    if (i < n) {
        const int e = t.vals[i];
        t.leaf_elem[i] = e;
        t.box_lo[n - 1 + i] = t.elem_lo[e];
        t.box_up[n - 1 + i] = t.elem_up[e];
    }
    if (i == 0) t.parent[0] = -1;
    if (i >= n - 1) return;
    t.flags[i] = 0u;
    const unsigned long long* K = t.keys;
    const int d = (karras_delta(K, n, i, i + 1) - karras_delta(K, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = karras_delta(K, n, i, i - d);
    int lmax = 2;
    while (karras_delta(K, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int s = lmax >> 1; s >= 1; s >>= 1)
        if (karras_delta(K, n, i, i + (l + s) * d) > dmin) l += s;
    const int j = i + l * d;
    const int dnode = karras_delta(K, n, i, j);
    int sp = 0;
    for (int div = 2;; div <<= 1) {
        const int s = (l + div - 1) / div;
        if (karras_delta(K, n, i, i + (sp + s) * d) > dnode) sp += s;
        if (s <= 1) break;
    }
    const int gamma = i + sp * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const int left = (lo == gamma) ? (n - 1 + gamma) : gamma;
    const int right = (hi == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
    t.left[i] = left;
    t.right[i] = right;
    t.parent[left] = i;
    t.parent[right] = i;
    t.node4[4 * i + 0].w = __int_as_float(left);
    t.node4[4 * i + 2].w = __int_as_float(right);
}

// Writes node `c`'s box into its parent's record (left or right slot).
ADMM_DEV void store_in_parent(const BvhDev& t, int c, float4 lo, float4 up) {
    const int p = t.parent[c];
    if (p < 0) return;
    const int slot = (t.left[p] == c) ? 0 : 2;
    float4* r = t.node4 + 4 * p + slot;
    const float idx = __ldcg(&r[0].w);
    __stcg(&r[0], make_float4(lo.x, lo.y, lo.z, idx));
    __stcg(&r[1], make_float4(up.x, up.y, up.z, 0.f));
}

// Refit of an existing tree: recompute the sorted leaves' boxes from the
// current positions and clear the arrival counters (k_refit follows).
template <int NV>
__global__ void __launch_bounds__(256) k_leaf_refresh(const float4* __restrict__ x, const int* __restrict__ elems,
                                                     int elem_stride, BvhDev t) {
    ADMM_PDL_PROLOGUE();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = t.n;
    if (k >= n) return;
    const int e = t.leaf_elem[k];
    float4 lo = f4(1e32f, 1e32f, 1e32f), up = f4(-1e32f, -1e32f, -1e32f);
#pragma unroll
    for (int j = 0; j < NV; j++) box_add(lo, up, x[elems[e * elem_stride + j]]);
    t.box_lo[n - 1 + k] = lo;
    t.box_up[n - 1 + k] = up;
    if (k < n - 1) t.flags[k] = 0u;
}

// Bottom-up refit: the second child to arrive at a node merges the boxes.
__global__ void __launch_bounds__(256) k_refit(BvhDev t) {
    ADMM_PDL_PROLOGUE();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = t.n;
    if (k >= n || n < 2) return;
    int node = n - 1 + k;
    store_in_parent(t, node, t.box_lo[node], t.box_up[node]);
    int p = t.parent[node];
    for (int guard = 0; p >= 0; guard++) {
        if (guard >= n) {  // deeper than any valid tree: malformed, stop
            t.flags[0] = 0x80000000u;
            return;
        }
        __threadfence();
        const unsigned old = atomicAdd(&t.flags[p], 1u);
        if (old == 0u) return;
        __threadfence();  // acquire: the sibling published its box before its atomic
        const float4 al = __ldcg(&t.node4[4 * p + 0]), au = __ldcg(&t.node4[4 * p + 1]);
        const float4 bl = __ldcg(&t.node4[4 * p + 2]), bu = __ldcg(&t.node4[4 * p + 3]);
        const float4 lo = f4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z));
        const float4 up = f4(fmaxf(au.x, bu.x), fmaxf(au.y, bu.y), fmaxf(au.z, bu.z));
        __stcg(&t.box_lo[p], lo);
        __stcg(&t.box_up[p], up);
        store_in_parent(t, p, lo, up);
        node = p;
        p = t.parent[p];
    }
}

// --------------------------- narrow phase -----------------------------------
struct NpResult {
    float dist;
    float bary[3];
    float c0[3], c1[3];
};

ADMM_DEV float ndot(float ax, float ay, float az, float bx, float by, float bz) {
    return fadd(fadd(fmul(ax, bx), fmul(ay, by)), fmul(az, bz));
}

// dcdPT region 0 (dist_g.cuh:29-252); returns false outside region 0.
ADMM_DEV bool narrow_pt(float4 P, float4 T0, float4 T1, float4 T2, NpResult& r) {
    const float dx = fsub(T0.x, P.x), dy = fsub(T0.y, P.y), dz = fsub(T0.z, P.z);
    const float e0x = fsub(T1.x, T0.x), e0y = fsub(T1.y, T0.y), e0z = fsub(T1.z, T0.z);
    const float e1x = fsub(T2.x, T0.x), e1y = fsub(T2.y, T0.y), e1z = fsub(T2.z, T0.z);
    const float a00 = ndot(e0x, e0y, e0z, e0x, e0y, e0z);
    const float a01 = ndot(e0x, e0y, e0z, e1x, e1y, e1z);
    const float a11 = ndot(e1x, e1y, e1z, e1x, e1y, e1z);
    const float b0 = ndot(dx, dy, dz, e0x, e0y, e0z);
    const float b1 = ndot(dx, dy, dz, e1x, e1y, e1z);
    const float det = fmaxf(fsub(fmul(a00, a11), fmul(a01, a01)), 0.f);
    float s = fsub(fmul(a01, b1), fmul(a11, b0));
    float t = fsub(fmul(a01, b0), fmul(a00, b1));
    if (!(fadd(s, t) <= det) || s < 0.f || t < 0.f) return false;
    s = fdiv(s, det);
    t = fdiv(t, det);
    r.c0[0] = P.x; r.c0[1] = P.y; r.c0[2] = P.z;
    r.c1[0] = fadd(fadd(T0.x, fmul(s, e0x)), fmul(t, e1x));
    r.c1[1] = fadd(fadd(T0.y, fmul(s, e0y)), fmul(t, e1y));
    r.c1[2] = fadd(fadd(T0.z, fmul(s, e0z)), fmul(t, e1z));
    const float qx = fsub(r.c0[0], r.c1[0]), qy = fsub(r.c0[1], r.c1[1]), qz = fsub(r.c0[2], r.c1[2]);
    r.dist = fsqrt(ndot(qx, qy, qz, qx, qy, qz));
    r.bary[0] = fsub(fsub(1.f, s), t);
    r.bary[1] = s;
    r.bary[2] = t;
    return true;
}

// dcdEE region 0 (dist_g.cuh:257-513).
ADMM_DEV bool narrow_ee(float4 P0, float4 P1, float4 Q0, float4 Q1, NpResult& r) {
    const float ux = fsub(P1.x, P0.x), uy = fsub(P1.y, P0.y), uz = fsub(P1.z, P0.z);
    const float vx = fsub(Q1.x, Q0.x), vy = fsub(Q1.y, Q0.y), vz = fsub(Q1.z, Q0.z);
    const float wx = fsub(P0.x, Q0.x), wy = fsub(P0.y, Q0.y), wz = fsub(P0.z, Q0.z);
    const float a = ndot(ux, uy, uz, ux, uy, uz);
    const float b = ndot(ux, uy, uz, vx, vy, vz);
    const float c = ndot(vx, vy, vz, vx, vy, vz);
    const float d = ndot(ux, uy, uz, wx, wy, wz);
    const float e = ndot(vx, vy, vz, wx, wy, wz);
    const float det = fsub(fmul(a, c), fmul(b, b));
    if (!(det > 0.f)) return false;
    const float bte = fmul(b, e), ctd = fmul(c, d);
    if (bte <= ctd) return false;
    float s = fsub(bte, ctd);
    if (s >= det) return false;
    const float ate = fmul(a, e), btd = fmul(b, d);
    if (ate <= btd) return false;
    float t = fsub(ate, btd);
    if (t >= det) return false;
    s = fdiv(s, det);
    t = fdiv(t, det);
    r.bary[0] = s;
    r.bary[1] = t;
    r.bary[2] = -10.f;
    r.c0[0] = fadd(P0.x, fmul(s, ux)); r.c0[1] = fadd(P0.y, fmul(s, uy)); r.c0[2] = fadd(P0.z, fmul(s, uz));
    r.c1[0] = fadd(Q0.x, fmul(t, vx)); r.c1[1] = fadd(Q0.y, fmul(t, vy)); r.c1[2] = fadd(Q0.z, fmul(t, vz));
    const float qx = fsub(r.c0[0], r.c1[0]), qy = fsub(r.c0[1], r.c1[1]), qz = fsub(r.c0[2], r.c1[2]);
    r.dist = fsqrt(ndot(qx, qy, qz, qx, qy, qz));
    return true;
}

// ---------------------------------------------------------------------------
// The CPU backend's closest points (ProximalQuery::narrow_PT / narrow_EE,
// narrow_phase.cpp:376-469, through Eberly's queries of distPT.h / distEE.h):
// every region, in the same operation order as the FP32 reference, so that the
// accepted sets agree bit for bit.  Point-triangle: the minimiser of
// |t0 + s e0 + t e1 - p|^2 on the triangle, chosen by the signs of s, t and
// s + t - det; edge-edge: the minimiser over [0,1]^2 by the signs of
// b e - c d and a e - b d, or along the square's edges for parallel segments.
// ---------------------------------------------------------------------------
ADMM_DEV float clamp_ratio(float n, float a) { return n <= 0.f ? 0.f : (n >= a ? 1.f : fdiv(n, a)); }

ADMM_DEV void closest_pt_all(float4 P, float4 T0, float4 T1, float4 T2, NpResult& r) {
    const float dx = fsub(T0.x, P.x), dy = fsub(T0.y, P.y), dz = fsub(T0.z, P.z);
    const float e0x = fsub(T1.x, T0.x), e0y = fsub(T1.y, T0.y), e0z = fsub(T1.z, T0.z);
    const float e1x = fsub(T2.x, T0.x), e1y = fsub(T2.y, T0.y), e1z = fsub(T2.z, T0.z);
    const float a00 = ndot(e0x, e0y, e0z, e0x, e0y, e0z);
    const float a01 = ndot(e0x, e0y, e0z, e1x, e1y, e1z);
    const float a11 = ndot(e1x, e1y, e1z, e1x, e1y, e1z);
    const float b0 = ndot(dx, dy, dz, e0x, e0y, e0z);
    const float b1 = ndot(dx, dy, dz, e1x, e1y, e1z);
    const float dd = fsub(fmul(a00, a11), fmul(a01, a01));
    const float det = dd < 0.f ? 0.f : dd;
    float s = fsub(fmul(a01, b1), fmul(a11, b0));
    float t = fsub(fmul(a01, b0), fmul(a00, b1));
    // the minimiser on an edge s = 0 (over t) or t = 0 (over s) from the sign of b
    const float on_t = b1 >= 0.f ? 0.f : (-b1 >= a11 ? 1.f : fdiv(-b1, a11));
    const float on_s = b0 >= 0.f ? 0.f : (-b0 >= a00 ? 1.f : fdiv(-b0, a00));
    if (fadd(s, t) <= det) {
        if (s < 0.f) {
            if (t < 0.f && b0 < 0.f) {
                t = 0.f;
                s = -b0 >= a00 ? 1.f : fdiv(-b0, a00);
            } else {
                s = 0.f;
                t = on_t;
            }
        } else if (t < 0.f) {
            t = 0.f;
            s = on_s;
        } else {
            s = fdiv(s, det);
            t = fdiv(t, det);
        }
    } else {
        const float den = fadd(fsub(a00, fmul(2.f, a01)), a11);
        if (s < 0.f) {
            const float q0 = fadd(a01, b0), q1 = fadd(a11, b1);
            if (q1 > q0) {
                const float num = fsub(q1, q0);
                if (num >= den) { s = 1.f; t = 0.f; }
                else { s = fdiv(num, den); t = fsub(1.f, s); }
            } else {
                s = 0.f;
                t = q1 <= 0.f ? 1.f : (b1 >= 0.f ? 0.f : fdiv(-b1, a11));
            }
        } else if (t < 0.f) {
            const float q0 = fadd(a01, b1), q1 = fadd(a00, b0);
            if (q1 > q0) {
                const float num = fsub(q1, q0);
                if (num >= den) { t = 1.f; s = 0.f; }
                else { t = fdiv(num, den); s = fsub(1.f, t); }
            } else {
                t = 0.f;
                s = q1 <= 0.f ? 1.f : (b0 >= 0.f ? 0.f : fdiv(-b0, a00));
            }
        } else {
            const float num = fsub(fsub(fadd(a11, b1), a01), b0);
            if (num <= 0.f) { s = 0.f; t = 1.f; }
            else if (num >= den) { s = 1.f; t = 0.f; }
            else { s = fdiv(num, den); t = fsub(1.f, s); }
        }
    }
    r.c0[0] = P.x; r.c0[1] = P.y; r.c0[2] = P.z;
    r.c1[0] = fadd(fadd(T0.x, fmul(s, e0x)), fmul(t, e1x));
    r.c1[1] = fadd(fadd(T0.y, fmul(s, e0y)), fmul(t, e1y));
    r.c1[2] = fadd(fadd(T0.z, fmul(s, e0z)), fmul(t, e1z));
    const float qx = fsub(r.c0[0], r.c1[0]), qy = fsub(r.c0[1], r.c1[1]), qz = fsub(r.c0[2], r.c1[2]);
    r.dist = fsqrt(ndot(qx, qy, qz, qx, qy, qz));
    r.bary[0] = fsub(fsub(1.f, s), t);
    r.bary[1] = s;
    r.bary[2] = t;
}

ADMM_DEV void closest_ee_all(float4 P0, float4 P1, float4 Q0, float4 Q1, NpResult& r) {
    const float ux = fsub(P1.x, P0.x), uy = fsub(P1.y, P0.y), uz = fsub(P1.z, P0.z);
    const float vx = fsub(Q1.x, Q0.x), vy = fsub(Q1.y, Q0.y), vz = fsub(Q1.z, Q0.z);
    const float wx = fsub(P0.x, Q0.x), wy = fsub(P0.y, Q0.y), wz = fsub(P0.z, Q0.z);
    const float a = ndot(ux, uy, uz, ux, uy, uz);
    const float b = ndot(ux, uy, uz, vx, vy, vz);
    const float c = ndot(vx, vy, vz, vx, vy, vz);
    const float d = ndot(ux, uy, uz, wx, wy, wz);
    const float e = ndot(vx, vy, vz, wx, wy, wz);
    const float det = fsub(fmul(a, c), fmul(b, b));
    float s = 0.f, t = 0.f;
    if (det > 0.f) {
        const float bte = fmul(b, e), ctd = fmul(c, d);
        if (bte <= ctd) {
            if (e <= 0.f) {
                const float nd = -d;
                s = nd >= a ? 1.f : (nd > 0.f ? fdiv(nd, a) : 0.f);
            } else if (e < c) {
                t = fdiv(e, c);
            } else {
                t = 1.f;
                const float bmd = fsub(b, d);
                s = bmd >= a ? 1.f : (bmd > 0.f ? fdiv(bmd, a) : 0.f);
            }
        } else {
            s = fsub(bte, ctd);
            if (s >= det) {
                const float bpe = fadd(b, e);
                if (bpe <= 0.f) {
                    const float nd = -d;
                    s = nd <= 0.f ? 0.f : (nd < a ? fdiv(nd, a) : 1.f);
                } else if (bpe < c) {
                    s = 1.f;
                    t = fdiv(bpe, c);
                } else {
                    t = 1.f;
                    const float bmd = fsub(b, d);
                    s = bmd <= 0.f ? 0.f : (bmd < a ? fdiv(bmd, a) : 1.f);
                }
            } else {
                const float ate = fmul(a, e), btd = fmul(b, d);
                if (ate <= btd) {
                    s = clamp_ratio(-d, a);
                } else {
                    t = fsub(ate, btd);
                    if (t >= det) {
                        t = 1.f;
                        s = clamp_ratio(fsub(b, d), a);
                    } else {
                        s = fdiv(s, det);
                        t = fdiv(t, det);
                    }
                }
            }
        }
    } else if (e <= 0.f) {
        s = clamp_ratio(-d, a);
    } else if (e >= c) {
        t = 1.f;
        s = clamp_ratio(fsub(b, d), a);
    } else {
        t = fdiv(e, c);
    }
    r.bary[0] = s;
    r.bary[1] = t;
    r.bary[2] = -10.f;
    r.c0[0] = fadd(P0.x, fmul(s, ux)); r.c0[1] = fadd(P0.y, fmul(s, uy)); r.c0[2] = fadd(P0.z, fmul(s, uz));
    r.c1[0] = fadd(Q0.x, fmul(t, vx)); r.c1[1] = fadd(Q0.y, fmul(t, vy)); r.c1[2] = fadd(Q0.z, fmul(t, vz));
    const float qx = fsub(r.c0[0], r.c1[0]), qy = fsub(r.c0[1], r.c1[1]), qz = fsub(r.c0[2], r.c1[2]);
    r.dist = fsqrt(ndot(qx, qy, qz, qx, qy, qz));
}

ADMM_DEV bool box_overlap(float4 llo, float4 lup, float4 rlo, float4 rup, float gap) {
    if ((rlo.x - lup.x) >= gap || (llo.x - rup.x) >= gap) return false;
    if ((rlo.y - lup.y) >= gap || (llo.y - rup.y) >= gap) return false;
    if ((rlo.z - lup.z) >= gap || (llo.z - rup.z) >= gap) return false;
    return true;
}

// convert_DCD_info_kernel (contact_solver.cu:118-154) for one accepted pair.
ADMM_DEV void write_contact(const DevScene& s, int slot, int4 ids, const NpResult& r, bool ee) {
    const float4 v0 = s.x[ids.x], v1 = s.x[ids.y], v2 = s.x[ids.z], v3 = s.x[ids.w];
    s.pairs[slot] = ids;
    s.point[slot] = f4(0.5f * (r.c0[0] + r.c1[0]), 0.5f * (r.c0[1] + r.c1[1]), 0.5f * (r.c0[2] + r.c1[2]));
    float4 bary;
    float nx, ny, nz;
    if (ee) {
        bary = make_float4(1.f - r.bary[0], r.bary[0], r.bary[1] - 1.f, -r.bary[1]);
        const float4 a = sub3(v1, v0), b = sub3(v3, v2);
        nx = a.y * b.z - a.z * b.y; ny = a.z * b.x - a.x * b.z; nz = a.x * b.y - a.y * b.x;
    } else {
        bary = make_float4(1.f, -r.bary[0], -r.bary[1], -r.bary[2]);
        const float4 a = sub3(v2, v1), b = sub3(v3, v1);
        nx = a.y * b.z - a.z * b.y; ny = a.z * b.x - a.x * b.z; nz = a.x * b.y - a.y * b.x;
    }
    const float nn = nx * nx + ny * ny + nz * nz;
    if (nn > 0.f) {
        const float inv = 1.f / sqrtf(nn);
        nx *= inv; ny *= inv; nz *= inv;
    }
    float hcn = (r.c0[0] - r.c1[0]) * nx + (r.c0[1] - r.c1[1]) * ny + (r.c0[2] - r.c1[2]) * nz;
    if (hcn < 0.f) {
        nx = -nx; ny = -ny; nz = -nz;
        hcn = -hcn;
    }
    s.bary[slot] = bary;
    s.nrm[slot] = make_float4(nx, ny, nz, hcn - s.thickness);
}

// --------------------------- traversal --------------------------------------
// VF: query q = surface vertex sv[q] against the face tree (lbvh.cu:1693-1748).
template <bool WRITE>
__global__ void __launch_bounds__(128) k_dcd_vf(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= s.nsv) return;
    const BvhDev& t = s.bf;
    const int v = s.sv[q];
    const float4 P = s.x[v];
    const float gap = s.thickness;
    int count = 0;
    const int base = WRITE ? s.qoff[q] : 0;
    int stack[kStackDepth];
    int sp = 0;
    const int n = t.n;
    auto visit = [&](int node, float4 blo, float4 bup) -> bool {  // true: push the (internal) node
        if (!box_overlap(P, P, blo, bup, gap)) return false;
        if (node < n - 1) return true;
        const int f = t.leaf_elem[node - (n - 1)];
        const int4 tri = s.st[f];
        if (v == tri.x || v == tri.y || v == tri.z) return false;
        NpResult r;
        if (narrow_pt(P, s.x[tri.x], s.x[tri.y], s.x[tri.z], r) && r.dist < gap && r.dist >= 0.f) {
            if (WRITE) {
                const int slot = base + count;
                if (slot < s.cap) write_contact(s, slot, make_int4(v, tri.x, tri.y, tri.z), r, false);
            }
            count++;
        }
        return false;
    };
    if (n == 1) {
        visit(0, t.box_lo[0], t.box_up[0]);
    } else if (n > 1) {
        stack[sp++] = 0;
        for (int pops = 0; sp > 0; pops++) {
            if (pops > 2 * n) {  // more pops than nodes: malformed tree, stop
                s.err[1] = 1;
                break;
            }
            const int node = stack[--sp];
            const float4* rec = t.node4 + 4 * node;
            const float4 ll = rec[0], lu = rec[1], rl = rec[2], ru = rec[3];
            const int l = __float_as_int(ll.w), r = __float_as_int(rl.w);
            if (visit(l, ll, lu)) {
                if (sp < kStackDepth) stack[sp++] = l;
                else s.err[1] = 1;
            }
            if (visit(r, rl, ru)) {
                if (sp < kStackDepth) stack[sp++] = r;
                else s.err[1] = 1;
            }
        }
    }
    if (!WRITE) s.qcount[q] = count;
}

// EE: query e = surface edge against the edge tree; only edges with a larger
// index that share no vertex (lbvh.cu:1750-1813).
template <bool WRITE>
__global__ void __launch_bounds__(128) k_dcd_ee(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= s.nse) return;
    const BvhDev& t = s.be;
    const int2 ed = s.se[e];
    const float4 A0 = s.x[ed.x], A1 = s.x[ed.y];
    float4 lo = f4(1e32f, 1e32f, 1e32f), up = f4(-1e32f, -1e32f, -1e32f);
    box_add(lo, up, A0);
    box_add(lo, up, A1);
    const float gap = s.thickness;
    int count = 0;
    const int base = WRITE ? s.qoff[s.nsv + e] : 0;
    int stack[kStackDepth];
    int sp = 0;
    const int n = t.n;
    auto visit = [&](int node, float4 blo, float4 bup) -> bool {
        if (!box_overlap(lo, up, blo, bup, gap)) return false;
        if (node < n - 1) return true;
        const int o = t.leaf_elem[node - (n - 1)];
        if (o <= e) return false;
        const int2 od = s.se[o];
        if (ed.x == od.x || ed.x == od.y || ed.y == od.x || ed.y == od.y) return false;
        NpResult r;
        if (narrow_ee(A0, A1, s.x[od.x], s.x[od.y], r) && r.dist < gap && r.dist >= 0.f) {
            if (WRITE) {
                const int slot = base + count;
                if (slot < s.cap) write_contact(s, slot, make_int4(ed.x, ed.y, od.x, od.y), r, true);
            }
            count++;
        }
        return false;
    };
    if (n == 1) {
        visit(0, t.box_lo[0], t.box_up[0]);
    } else if (n > 1) {
        stack[sp++] = 0;
        for (int pops = 0; sp > 0; pops++) {
            if (pops > 2 * n) {  // more pops than nodes: malformed tree, stop
                s.err[1] = 1;
                break;
            }
            const int node = stack[--sp];
            const float4* rec = t.node4 + 4 * node;
            const float4 ll = rec[0], lu = rec[1], rl = rec[2], ru = rec[3];
            const int l = __float_as_int(ll.w), r = __float_as_int(rl.w);
            if (visit(l, ll, lu)) {
                if (sp < kStackDepth) stack[sp++] = l;
                else s.err[1] = 1;
            }
            if (visit(r, rl, ru)) {
                if (sp < kStackDepth) stack[sp++] = r;
                else s.err[1] = 1;
            }
        }
    }
    if (!WRITE) s.qcount[s.nsv + e] = count;
}

// nc = min(total, cap); overflow flag.
__global__ void k_set_count(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int raw = *s.nc_raw;
    *s.nc = raw < s.cap ? raw : s.cap;
    if (raw > s.cap) s.err[0] = 1;
}

}  // namespace admm
