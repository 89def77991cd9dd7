// learn.cuh -- the learned global step (global_solver 3), an addition
// with no counterpart in the reference.  It replaces the jacobi_iter Jacobi sweeps
// of an ADMM iteration (cu_jacobi_global, jacobi_solver.cu:141-180, called from
// admm_impl_gpu.cu:364) by K sweeps of a second-order iteration
//
//     x_{k+1} = x_k + omega_k m (b - A x_k) + beta_k (x_k - x_{k-1}),   beta_0 = 0,
//
// started from the warm start x_0 = x + theta (x - x_last), where x is the iterate
// the global step receives and x_last the one the previous global step of the
// substep received (no warm start in the first global step of a substep).  m
// (per dynamic vertex, scaling the isotropic system A (x) I3) and theta (per
// dynamic vertex) come from the learned network; the K pairs (omega_k, beta_k)
// are trained with it.  omega = 1, beta = 0, theta = 0 and m = 1 / a_ii is the
// Jacobi sweep itself.
//
// The judge: a solve fails when its final residual |b - A x_K| is larger than the
// received iterate's |b - A x_c| and above 1e-5 |b| (below that it is FP32 rounding
// noise of b - A x, where the comparison decides nothing).  Judging against the received
// iterate, not x_0, also catches a warm start that made things worse.  The sums: the
// first sweep adds up |b - A x_0|^2 and |b|^2, the judge's pass (k_ljudge) |b - A x_K|^2;
// the judge's pass also keeps A x_K, which is A x_c of the substep's next global step (the
// local and contact steps in between do not move x), so the first sweep sums
// |b - A x_c|^2 with the new b without a second pass over A.  In the substep's first
// global step x_0 = x_c.
// The warm start restarts adaptively (the function-value restart of accelerated methods,
// O'Donoghue and Candes 2015, on the residual norm): once a warm start raised the
// residual, |b - A x_0| > |b - A x_c|, it stays off until the substep's next first global
// step.  A failed solve is replaced on the device by the plain one: x <- x_c (kept in xl),
// then the jacobi_iter Jacobi sweeps and a pass that refreshes A x, in the body of a
// conditional (IF) node of the substep graph whose condition k_ldecide sets; the rest of
// the substep goes on.
//
// Buffers: x_k lives in {x, jac0, jac1}[(s0 + k) % 3] with s0 = -K mod 3, so that x_K
// ends in x; k_rhs_learn writes x_0 (x_c or its warm start) into the buffer of k = 0.
#pragma once
#include "kernels.cuh"

namespace admm {

constexpr int kLearnMaxSweeps = 32;

struct LearnDev {
    const float* minv = nullptr;   // [nd] m_i
    const float* theta = nullptr;  // [nd] warm-start coefficient
    float4* xl = nullptr;          // [nd] x received by the previous global step
    float4* ax = nullptr;          // [nd] A x after the last global step (judge's pass or fallback)
    double* part = nullptr;        // [3 x blocks] block partials of |r_0|^2, |r_K|^2 and |b|^2
    double* part_c = nullptr;      // [blocks] block partials of |r_c|^2 (first sweep)
    int blocks = 0;                // grid of the sweeps and the judge
    int rblocks = 0;               // grid of k_rhs_learn
    unsigned long long* stats = nullptr;  // [4] solves judged, solves failed (device counters)
    int* fail = nullptr;           // [1] 1 when the solve judged last failed (read by eager substeps)
    int* warm = nullptr;           // [1] 1 while the warm start is on in this substep
};

// Right-hand side (as k_rhs) plus the start of the solve: xl <- x_c (the received x),
// x0buf <- x_c + theta (x_c - xl_old) while L.warm is set, else x_c (not rewritten when
// x0buf is x itself).  extrap = 0 in the substep's first global step, where the warm start
// is switched on for the substep.
template <int T, bool SAVE_PREV>
__global__ void __launch_bounds__(kVertThreads) k_rhs_learn(DevScene s, LearnDev L, int extrap,
                                                            float4* __restrict__ x0buf) {
    ADMM_PDL_TRIGGER();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= s.R.nslices) return;
    EllRowPf<T, true> r;
    r.load(s.R, w, lane);
    const int i = r.row;
    const bool own = i < s.nd, c = own && s.contact;
    const float wc = c ? __ldg(&s.dt2wc[i]) : 0.f;
    const float th = own && extrap ? __ldg(&L.theta[i]) : 0.f;
    ADMM_PDL_WAIT();
    if (!extrap && blockIdx.x == 0 && threadIdx.x == 0) *L.warm = 1;  // nobody reads it in this launch
    const bool warm = extrap && *L.warm;
    const float4 z = f4(0.f, 0.f, 0.f);
    const float4 m = own ? s.mxt[i] : z, p = c ? s.p[i] : z, x0 = c ? s.x0[i] : z, uc = c ? s.uc[i] : z;
    const float4 xi = own ? s.x[i] : z;
    const float4 xo = own && warm ? L.xl[i] : z;
    const float4 acc = r.sum(s.R, s.y, lane);
    if (lane >= 32 / T || !own) return;
    s.b[i] = rhs_value(s, acc, m, p, x0, uc, wc);
    if (SAVE_PREV) s.xprev[i] = xi;
    L.xl[i] = xi;
    if (warm)
        x0buf[i] = f4(fmaf(th, xi.x - xo.x, xi.x), fmaf(th, xi.y - xo.y, xi.y), fmaf(th, xi.z - xo.z, xi.z));
    else if (x0buf != s.x)
        x0buf[i] = xi;
}

// One learned sweep k: dst = src + omega m (b - A src) + beta (src - prev); the first
// sweep (FIRST) also writes the block partials of |b - A x_0|^2 into L.part[0..) and of
// |b|^2 into L.part[2 blocks..), and, outside the substep's first global step (extrap),
// of |b - A x_c|^2 into L.part_c, A x_c from L.ax.
// The sweep and the judge's pass are capped at 40 registers (12 blocks per SM) for the same
// reason as k_jacobi (batch: 65.4 -> 56.0 us per learned sweep in the step graph).
template <int T, bool FIRST>
__global__ void __launch_bounds__(kVertThreads, 12) k_lsweep(DevScene s, LearnDev L, const float4* __restrict__ src,
                                                         const float4* __restrict__ prev, float4* __restrict__ dst,
                                                         float omega, float beta, int extrap) {
    ADMM_PDL_TRIGGER();
    __shared__ double sh[kVertThreads / 32];
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double rr = 0.0, bb = 0.0, rc = 0.0;
    if (w < s.A.nslices) {
        EllRowPf<T> r;
        r.load(s.A, w, lane);
        const int i = r.row;
        const bool own = i < s.nd;
        const float d = own ? __ldg(&s.a_diag[i]) : 1.f;
        const float mi = own ? __ldg(&L.minv[i]) : 0.f;
        ADMM_PDL_WAIT();
        const float4 zz = f4(0.f, 0.f, 0.f);
        const float4 bi = own ? s.b[i] : zz, xi = own ? src[i] : zz;
        const float4 xp = own && !FIRST ? prev[i] : xi;
        const float4 acc = r.sum(s.A, src, lane);
        if (lane < 32 / T && own) {
            const float rx = bi.x - fmaf(d, xi.x, acc.x), ry = bi.y - fmaf(d, xi.y, acc.y),
                        rz = bi.z - fmaf(d, xi.z, acc.z);
            const float ox = omega * mi, bx = beta;
            dst[i] = f4(fmaf(ox, rx, fmaf(bx, xi.x - xp.x, xi.x)), fmaf(ox, ry, fmaf(bx, xi.y - xp.y, xi.y)),
                        fmaf(ox, rz, fmaf(bx, xi.z - xp.z, xi.z)));
            if (FIRST) {
                rr = (double)rx * rx + (double)ry * ry + (double)rz * rz;
                bb = (double)bi.x * bi.x + (double)bi.y * bi.y + (double)bi.z * bi.z;
                if (extrap) {
                    const float4 ai = L.ax[i];
                    const float cx = bi.x - ai.x, cy = bi.y - ai.y, cz = bi.z - ai.z;
                    rc = (double)cx * cx + (double)cy * cy + (double)cz * cz;
                }
            }
        }
    } else {
        ADMM_PDL_WAIT();
    }
    if (FIRST) {
        rr = block_sum(rr, sh);
        bb = block_sum(bb, sh);
        if (extrap) rc = block_sum(rc, sh);
        if (threadIdx.x == 0) {
            L.part[blockIdx.x] = rr;
            L.part[2 * L.blocks + blockIdx.x] = bb;
            if (extrap) L.part_c[blockIdx.x] = rc;
        }
    }
}

// The judge's pass over x (= x_K, or the plain solve's result in a fallback): block
// partials of |b - A x|^2 into L.part[blocks..) and L.ax <- A x.
template <int T>
__global__ void __launch_bounds__(kVertThreads, 12) k_ljudge(DevScene s, LearnDev L) {
    ADMM_PDL_TRIGGER();
    __shared__ double sh[kVertThreads / 32];
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double rr = 0.0;
    if (w < s.A.nslices) {
        EllRowPf<T> r;
        r.load(s.A, w, lane);
        const int i = r.row;
        const bool own = i < s.nd;
        const float d = own ? __ldg(&s.a_diag[i]) : 1.f;
        ADMM_PDL_WAIT();
        const float4 zz = f4(0.f, 0.f, 0.f);
        const float4 bi = own ? s.b[i] : zz, xi = own ? s.x[i] : zz;
        const float4 acc = r.sum(s.A, s.x, lane);
        if (lane < 32 / T && own) {
            const float4 a = f4(fmaf(d, xi.x, acc.x), fmaf(d, xi.y, acc.y), fmaf(d, xi.z, acc.z));
            L.ax[i] = a;
            const float rx = bi.x - a.x, ry = bi.y - a.y, rz = bi.z - a.z;
            rr = (double)rx * rx + (double)ry * ry + (double)rz * rz;
        }
    } else {
        ADMM_PDL_WAIT();
    }
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) L.part[L.blocks + blockIdx.x] = rr;
}

// One block of kDecideThreads: the partials summed in a fixed order (each thread a
// strided share, four loads in flight); a solve whose residual is above the received
// iterate's and above kJudgeFloor |b| counts as failed.  The decision goes to L.fail and,
// inside a graph, to the condition of the IF node that runs the plain solve.  A warm start
// that raised the residual switches the warm start off (without one, x_0 = x_c and the two
// sums agree).  first: the substep's first global step, where r_c = r_0.
constexpr double kJudgeFloor = 1e-5;
constexpr int kDecideThreads = 1024;
ADMM_DEV double strided_sum(const double* __restrict__ a, int n) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int k = threadIdx.x;
    for (; k + 3 * kDecideThreads < n; k += 4 * kDecideThreads) {
        s0 += a[k];
        s1 += a[k + kDecideThreads];
        s2 += a[k + 2 * kDecideThreads];
        s3 += a[k + 3 * kDecideThreads];
    }
    for (; k < n; k += kDecideThreads) s0 += a[k];
    return (s0 + s1) + (s2 + s3);
}

__global__ void __launch_bounds__(kDecideThreads) k_ldecide(LearnDev L, cudaGraphConditionalHandle cond, int in_graph,
                                                            int first) {
    ADMM_PDL_PROLOGUE();
    __shared__ double sh[kDecideThreads / 32];
    double e = strided_sum(L.part, L.blocks);
    double b = strided_sum(L.part + L.blocks, L.blocks);
    double c = strided_sum(L.part + 2 * L.blocks, L.blocks);
    double a = first ? 0.0 : strided_sum(L.part_c, L.blocks);
    e = block_sum(e, sh);
    b = block_sum(b, sh);
    c = block_sum(c, sh);
    a = block_sum(a, sh);
    if (threadIdx.x == 0) {
        if (first) a = e;
        const bool failed = !(b <= a || b <= kJudgeFloor * kJudgeFloor * c);
        L.stats[0] += 1ull;
        if (failed) L.stats[1] += 1ull;
        *L.fail = failed ? 1 : 0;
        if (e > a) *L.warm = 0;
        if (in_graph) cudaGraphSetConditional(cond, failed ? 1u : 0u);
    }
}

}  // namespace admm
