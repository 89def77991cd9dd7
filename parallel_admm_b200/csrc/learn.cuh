// learn.cuh -- the learned global step (global_solver 3), a north-star addition
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
// The judge: the first sweep sums |b - A x|^2 at the iterate x the step received
// (a second gather over the same matrix entries when a warm start moved x_0 away
// from it) and |b|^2, a last pass (k_ljudge) sums |b - A x_K|^2 while it moves x_K
// into x; k_ldecide counts the solve as failed when the residual is larger than the
// received iterate's and above 1e-5 |b| (below that it is FP32 rounding noise of
// b - A x, where the comparison decides nothing).  Judging against the received
// iterate, not x_0, also catches a warm start that made things worse.  The warm start
// restarts adaptively (the function-value restart of accelerated methods, O'Donoghue
// and Candes 2015, on the residual norm): once a warm start raised the residual,
// |b - A x_0| > |b - A x_c|, it stays off until the substep's next first global step.  A failed solve
// is replaced on the device by the plain one: x <- x as received (kept in xl), then
// the jacobi_iter Jacobi sweeps, in the body of a conditional (IF) node of the
// substep graph whose condition k_ldecide sets; the rest of the substep goes on.
#pragma once
#include "kernels.cuh"

namespace admm {

constexpr int kLearnMaxSweeps = 32;

struct LearnDev {
    const float* minv = nullptr;   // [nd] m_i
    const float* theta = nullptr;  // [nd] warm-start coefficient
    float4* xl = nullptr;          // [nd] x received by the previous global step
    double* part = nullptr;        // [4 x blocks] block partials of |r_c|^2, |r_K|^2, |b|^2, |r_0|^2
                                   // (r_c at the received x, r_0 at the warm start x_0)
    int blocks = 0;                // grid of the sweeps and the judge
    unsigned long long* stats = nullptr;  // [4] solves judged, solves failed (device counters)
    int* fail = nullptr;           // [1] 1 when the solve judged last failed (read by eager substeps)
    int* warm = nullptr;           // [1] 1 while the warm start is on in this substep
};

// Right-hand side (as k_rhs) plus the warm start: xl <- x, x <- x + theta (x - xl_old)
// while L.warm is set (extrap = 0 in the first global step of a substep: xl only
// recorded, and the warm start switched on for the substep).
template <int T, bool SAVE_PREV>
__global__ void __launch_bounds__(kVertThreads) k_rhs_learn(DevScene s, LearnDev L, int extrap) {
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
    if (warm) s.x[i] = f4(fmaf(th, xi.x - xo.x, xi.x), fmaf(th, xi.y - xo.y, xi.y), fmaf(th, xi.z - xo.z, xi.z));
}

// One learned sweep k: dst = src + omega m (b - A src) + beta (src - prev); the first
// sweep (FIRST) also writes the block partials of |b - A x_c|^2 into L.part[0..), of
// |b|^2 into L.part[2 blocks..) and of |b - A src|^2 into L.part[3 blocks..), x_c the
// received iterate: xc (its copy in L.xl) when a warm start may have moved src, src
// itself otherwise (xc null).
template <int T, bool FIRST>
__global__ void __launch_bounds__(kVertThreads) k_lsweep(DevScene s, LearnDev L, const float4* __restrict__ src,
                                                         const float4* __restrict__ prev, float4* __restrict__ dst,
                                                         float omega, float beta, const float4* __restrict__ xc) {
    ADMM_PDL_TRIGGER();
    __shared__ double sh[kVertThreads / 32];
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double rr = 0.0, bb = 0.0, r0 = 0.0;
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
        float4 accc = acc;
        if (FIRST && xc) accc = r.sum(s.A, xc, lane);  // the prefetched entries, gathered at x_c
        if (lane < 32 / T && own) {
            const float rx = bi.x - fmaf(d, xi.x, acc.x), ry = bi.y - fmaf(d, xi.y, acc.y),
                        rz = bi.z - fmaf(d, xi.z, acc.z);
            const float ox = omega * mi, bx = beta;
            dst[i] = f4(fmaf(ox, rx, fmaf(bx, xi.x - xp.x, xi.x)), fmaf(ox, ry, fmaf(bx, xi.y - xp.y, xi.y)),
                        fmaf(ox, rz, fmaf(bx, xi.z - xp.z, xi.z)));
            if (FIRST) {
                const float4 ci = xc ? xc[i] : xi;
                const float cx = bi.x - fmaf(d, ci.x, accc.x), cy = bi.y - fmaf(d, ci.y, accc.y),
                            cz = bi.z - fmaf(d, ci.z, accc.z);
                rr = (double)cx * cx + (double)cy * cy + (double)cz * cz;
                bb = (double)bi.x * bi.x + (double)bi.y * bi.y + (double)bi.z * bi.z;
                r0 = (double)rx * rx + (double)ry * ry + (double)rz * rz;
            }
        }
    } else {
        ADMM_PDL_WAIT();
    }
    if (FIRST) {
        rr = block_sum(rr, sh);
        bb = block_sum(bb, sh);
        r0 = block_sum(r0, sh);
        if (threadIdx.x == 0) {
            L.part[blockIdx.x] = rr;
            L.part[2 * L.blocks + blockIdx.x] = bb;
            L.part[3 * L.blocks + blockIdx.x] = r0;
        }
    }
}

// The judge's pass: block partials of |b - A xk|^2 into L.part[blocks..); x <- xk
// (xk != x).
template <int T>
__global__ void __launch_bounds__(kVertThreads) k_ljudge(DevScene s, LearnDev L, const float4* __restrict__ xk) {
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
        const float4 bi = own ? s.b[i] : zz, xi = own ? xk[i] : zz;
        const float4 acc = r.sum(s.A, xk, lane);
        if (lane < 32 / T && own) {
            const float rx = bi.x - fmaf(d, xi.x, acc.x), ry = bi.y - fmaf(d, xi.y, acc.y),
                        rz = bi.z - fmaf(d, xi.z, acc.z);
            rr = (double)rx * rx + (double)ry * ry + (double)rz * rz;
            if (xk != s.x) s.x[i] = xi;
        }
    } else {
        ADMM_PDL_WAIT();
    }
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) L.part[L.blocks + blockIdx.x] = rr;
}

// One block: the partials summed in a fixed order; a solve whose residual is above the
// received iterate's and above kJudgeFloor |b| counts as failed.  The decision goes to L.fail and,
// inside a graph, to the condition of the IF node that runs the plain solve.  A warm start
// that raised the residual switches the warm start off (without one, x_0 = x_c and the
// two sums are equal bit for bit).
constexpr double kJudgeFloor = 1e-5;
__global__ void __launch_bounds__(256) k_ldecide(LearnDev L, cudaGraphConditionalHandle cond, int in_graph) {
    ADMM_PDL_PROLOGUE();
    __shared__ double sh[8];
    double a = 0.0, b = 0.0, c = 0.0, e = 0.0;
    for (int k = threadIdx.x; k < L.blocks; k += blockDim.x) {
        a += L.part[k];
        b += L.part[L.blocks + k];
        c += L.part[2 * L.blocks + k];
        e += L.part[3 * L.blocks + k];
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    c = block_sum(c, sh);
    e = block_sum(e, sh);
    if (threadIdx.x == 0) {
        const bool failed = !(b <= a || b <= kJudgeFloor * kJudgeFloor * c);
        L.stats[0] += 1ull;
        if (failed) L.stats[1] += 1ull;
        *L.fail = failed ? 1 : 0;
        if (e > a) *L.warm = 0;
        if (in_graph) cudaGraphSetConditional(cond, failed ? 1u : 0u);
    }
}

}  // namespace admm
