// learn.cu -- training of the learned global step (an addition with no
// reference counterpart): the loss of K unrolled sweeps of
//
//     x_0 = x_c + theta (x_c - x_l),
//     x_{k+1} = x_k + omega_k m (b - A x_k) + beta_k (x_k - x_{k-1})   (beta_0 = 0),
//
// L = (x_K - x*)^T A (x_K - x*) / ((x_c - x*)^T A (x_c - x*))
//     + mu |b - A x_K|^2 / |b - A x_c|^2   (mu = 0 unless set: the residual the judge checks),
// averaged over samples (b, x_c, x_l, x*) that plain runs produce, and its gradient with
// respect to omega, beta (per sweep), m and theta (per vertex) by the adjoint
// recursion (A symmetric, b - A x = -A (x - x*)):
//
//     g_K = 2 A (x_K - x*) / E_c + mu 2 A A (x_K - x*) / R_c,
//     g_k = (1 + beta_k) g_{k+1} - omega_k A (m g_{k+1}) - beta_{k+1} g_{k+2},
//     dL/domega_k = g_{k+1} . m r_k,   dL/dbeta_k = g_{k+1} . (x_k - x_{k-1}),
//     dL/dm_i = sum_k omega_k g_{k+1,i} . r_{k,i},   dL/dtheta_i = g_{0,i} . (x_c - x_l)_i.
//
// Also a conjugate-gradient solve of A x* = b (the converged solution of a
// sample).  One thread per row over a CSR copy of A (off-diagonal part plus
// diagonal); the per-sweep dot products are FP64 block partials summed in a
// fixed order, so a gradient is deterministic.  The FP64 restatement that the
// tests check these kernels against is in the oracle directory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <new>
#include <vector>

#include "admm_b200.h"

namespace {

constexpr int kT = 256;
constexpr int kParts = 296;  // blocks of the reduction kernels (2 x 148 SMs)
constexpr int kMaxK = 32;

inline int nblk(size_t n, int t) { return (int)((n + t - 1) / t); }

// out_i = (A v)_i over 3 columns
__device__ __forceinline__ void row_spmv(const int* __restrict__ start, const int* __restrict__ col,
                                         const float* __restrict__ val, const float* __restrict__ diag,
                                         const float* __restrict__ v, int i, float out[3]) {
    float a0 = diag[i] * v[3 * i], a1 = diag[i] * v[3 * i + 1], a2 = diag[i] * v[3 * i + 2];
    for (int e = start[i]; e < start[i + 1]; e++) {
        const int j = col[e];
        const float w = val[e];
        a0 = fmaf(w, v[3 * j], a0);
        a1 = fmaf(w, v[3 * j + 1], a1);
        a2 = fmaf(w, v[3 * j + 2], a2);
    }
    out[0] = a0;
    out[1] = a1;
    out[2] = a2;
}

// x0 = xc + theta (xc - xl)
__global__ void k_t_init(const float* __restrict__ xc, const float* __restrict__ xl, const float* __restrict__ th, int n,
                         float* __restrict__ x0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) x0[3 * i + c] = fmaf(th[i], xc[3 * i + c] - xl[3 * i + c], xc[3 * i + c]);
}

// r_k = b - A x_k; x_{k+1} = x_k + omega m r_k + beta (x_k - x_{k-1})
__global__ void k_t_sweep(const int* __restrict__ start, const int* __restrict__ col, const float* __restrict__ val,
                          const float* __restrict__ diag, const float* __restrict__ m, const float* __restrict__ b,
                          const float* __restrict__ xk, const float* __restrict__ xkm1, int n, float omega, float beta,
                          float* __restrict__ rk, float* __restrict__ xk1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float ax[3];
    row_spmv(start, col, val, diag, xk, i, ax);
    for (int c = 0; c < 3; c++) {
        const int q = 3 * i + c;
        const float r = b[q] - ax[c];
        rk[q] = r;
        xk1[q] = fmaf(omega * m[i], r, fmaf(beta, xk[q] - xkm1[q], xk[q]));
    }
}

// e = x - xs
__global__ void k_t_diff(const float* __restrict__ x, const float* __restrict__ xs, size_t cnt, float* __restrict__ e) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < cnt) e[t] = x[t] - xs[t];
}

// ae = A e, block partials of e . A e
__global__ void k_t_anorm2(const int* __restrict__ start, const int* __restrict__ col, const float* __restrict__ val,
                           const float* __restrict__ diag, const float* __restrict__ e, int n, float* __restrict__ ae,
                           double* __restrict__ part) {
    __shared__ double sh[kT];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float a[3];
        row_spmv(start, col, val, diag, e, i, a);
        for (int c = 0; c < 3; c++) {
            ae[3 * i + c] = a[c];
            acc += (double)a[c] * (double)e[3 * i + c];
        }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// block partials of v . v
__global__ void k_t_sq(const float* __restrict__ v, size_t cnt, double* __restrict__ part) {
    __shared__ double sh[kT];
    double acc = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += (size_t)gridDim.x * blockDim.x)
        acc += (double)v[t] * (double)v[t];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// g = s1 a (+ s2 c when c is given)
__global__ void k_t_seed(float* __restrict__ g, const float* __restrict__ a, const float* __restrict__ c, size_t cnt,
                         double s1, double s2) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    double v = (double)a[t] * s1;
    if (c) v += (double)c[t] * s2;
    g[t] = (float)v;
}

// One adjoint step k: gk = (1 + beta_k) g1 - omega_k A (m g1) - beta_{k+1} g2 (g2 may be
// null); partials of g1 . m r_k and g1 . (x_k - x_{k-1}); gm_i += omega_k g1_i . r_k,i.
__global__ void k_t_adjoint(const int* __restrict__ start, const int* __restrict__ col, const float* __restrict__ val,
                            const float* __restrict__ diag, const float* __restrict__ m, const float* __restrict__ g1,
                            const float* __restrict__ g2, const float* __restrict__ rk, const float* __restrict__ xk,
                            const float* __restrict__ xkm1, int n, float omega, float beta_k, float beta_k1,
                            float* __restrict__ gk, float* __restrict__ gm, double* __restrict__ part_o,
                            double* __restrict__ part_b) {
    __shared__ double sh[2 * kT];
    double ao = 0.0, ab = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        // A (m g1) row i
        float a0 = diag[i] * m[i] * g1[3 * i], a1 = diag[i] * m[i] * g1[3 * i + 1], a2 = diag[i] * m[i] * g1[3 * i + 2];
        for (int e = start[i]; e < start[i + 1]; e++) {
            const int j = col[e];
            const float w = val[e] * m[j];
            a0 = fmaf(w, g1[3 * j], a0);
            a1 = fmaf(w, g1[3 * j + 1], a1);
            a2 = fmaf(w, g1[3 * j + 2], a2);
        }
        const float amg[3] = {a0, a1, a2};
        float gmi = 0.f;
        for (int c = 0; c < 3; c++) {
            const int q = 3 * i + c;
            float g = fmaf(1.f + beta_k, g1[q], -omega * amg[c]);
            if (g2) g = fmaf(-beta_k1, g2[q], g);
            gk[q] = g;
            ao += (double)g1[q] * (double)m[i] * (double)rk[q];
            ab += (double)g1[q] * ((double)xk[q] - (double)xkm1[q]);
            gmi = fmaf(g1[q], rk[q], gmi);
        }
        gm[i] = fmaf(omega, gmi, gm[i]);
    }
    sh[threadIdx.x] = ao;
    sh[kT + threadIdx.x] = ab;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sh[threadIdx.x] += sh[threadIdx.x + o];
            sh[kT + threadIdx.x] += sh[kT + threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part_o[blockIdx.x] = sh[0];
        part_b[blockIdx.x] = sh[kT];
    }
}

// gth_i += g0_i . (xc - xl)_i
__global__ void k_t_theta(const float* __restrict__ g0, const float* __restrict__ xc, const float* __restrict__ xl, int n,
                          float* __restrict__ gth) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a = 0.f;
    for (int c = 0; c < 3; c++) a = fmaf(g0[3 * i + c], xc[3 * i + c] - xl[3 * i + c], a);
    gth[i] += a;
}

// ---- conjugate gradients (diag(A) preconditioned) for the converged solution ----
// r = b - A x, z = r / a, p = z; part = r . z
__global__ void k_cg_init(const int* __restrict__ start, const int* __restrict__ col, const float* __restrict__ val,
                          const float* __restrict__ diag, const float* __restrict__ b, const float* __restrict__ x, int n,
                          float* __restrict__ r, float* __restrict__ p, double* __restrict__ part) {
    __shared__ double sh[kT];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float a[3];
        row_spmv(start, col, val, diag, x, i, a);
        for (int c = 0; c < 3; c++) {
            const int q = 3 * i + c;
            const float rr = b[q] - a[c];
            r[q] = rr;
            p[q] = rr / diag[i];
            acc += (double)rr * (double)(rr / diag[i]);
        }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// q = A p, part = p . q
__global__ void k_cg_q(const int* __restrict__ start, const int* __restrict__ col, const float* __restrict__ val,
                       const float* __restrict__ diag, const float* __restrict__ p, int n, float* __restrict__ q,
                       double* __restrict__ part) {
    __shared__ double sh[kT];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float a[3];
        row_spmv(start, col, val, diag, p, i, a);
        for (int c = 0; c < 3; c++) {
            q[3 * i + c] = a[c];
            acc += (double)a[c] * (double)p[3 * i + c];
        }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// x += alpha p, r -= alpha q; part = r . r/a (new rz)
__global__ void k_cg_xr(const float* __restrict__ diag, const float* __restrict__ p, const float* __restrict__ q, int n,
                        double alpha, float* __restrict__ x, float* __restrict__ r, double* __restrict__ part) {
    __shared__ double sh[kT];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) {
            const int k = 3 * i + c;
            x[k] = (float)((double)x[k] + alpha * (double)p[k]);
            const float rr = (float)((double)r[k] - alpha * (double)q[k]);
            r[k] = rr;
            acc += (double)rr * (double)(rr / diag[i]);
        }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// p = r / a + beta p
__global__ void k_cg_p(const float* __restrict__ diag, const float* __restrict__ r, int n, double beta,
                       float* __restrict__ p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) p[3 * i + c] = (float)((double)(r[3 * i + c] / diag[i]) + beta * (double)p[3 * i + c]);
}

}  // namespace

struct AdmmLearn {
    int n = 0, nnz = 0;
    std::vector<void*> allocs;
    int *start = nullptr, *col = nullptr;
    float *val = nullptr, *diag = nullptr, *m = nullptr, *th = nullptr;
    float *b = nullptr, *xc = nullptr, *xl = nullptr, *xs = nullptr;
    float* X = nullptr;  // [(kMaxK + 1) * 3n] iterates
    float* Rk = nullptr; // [kMaxK * 3n] residuals
    float *g[3] = {nullptr, nullptr, nullptr}, *e = nullptr, *ae = nullptr;
    float* a2e = nullptr;  // A A e for the residual term
    double mu = 0.0;       // weight of the residual term
    float *gm = nullptr, *gth = nullptr;
    float *cr = nullptr, *cp = nullptr, *cq = nullptr;
    double* part = nullptr;  // [3 * kParts]
    cudaStream_t st = nullptr;
};

namespace {

template <class T>
int lalloc(AdmmLearn* L, T** p, size_t count) {
    if (count == 0) count = 1;
    if (cudaMalloc((void**)p, count * sizeof(T)) != cudaSuccess) return ADMM_ERR_OOM;
    L->allocs.push_back(*p);
    cudaMemset(*p, 0, count * sizeof(T));
    return ADMM_OK;
}

int sum_parts(AdmmLearn* L, const double* dev, int k, double* out) {
    std::vector<double> h(k);
    if (cudaMemcpyAsync(h.data(), dev, sizeof(double) * k, cudaMemcpyDeviceToHost, L->st) != cudaSuccess)
        return ADMM_ERR_CUDA;
    if (cudaStreamSynchronize(L->st) != cudaSuccess) return ADMM_ERR_CUDA;
    double s = 0.0;
    for (int i = 0; i < k; i++) s += h[i];
    *out = s;
    return ADMM_OK;
}

}  // namespace

extern "C" {

int admm_learn_create(int n, const int32_t* start, const int32_t* col, const float* val, const float* diag,
                      AdmmLearn** out) {
    if (!out || n <= 0 || !start || !diag) return ADMM_ERR_INVALID;
    *out = nullptr;
    const int nnz = start[n];
    if (nnz < 0 || (nnz > 0 && (!col || !val))) return ADMM_ERR_INVALID;
    AdmmLearn* L = new (std::nothrow) AdmmLearn;
    if (!L) return ADMM_ERR_OOM;
    L->n = n;
    L->nnz = nnz;
    const size_t N3 = 3 * (size_t)n;
    int rc = ADMM_OK;
    if ((rc = lalloc(L, &L->start, n + 1)) || (rc = lalloc(L, &L->col, nnz)) || (rc = lalloc(L, &L->val, nnz)) ||
        (rc = lalloc(L, &L->diag, n)) || (rc = lalloc(L, &L->m, n)) || (rc = lalloc(L, &L->th, n)) ||
        (rc = lalloc(L, &L->b, N3)) || (rc = lalloc(L, &L->xc, N3)) || (rc = lalloc(L, &L->xl, N3)) ||
        (rc = lalloc(L, &L->xs, N3)) || (rc = lalloc(L, &L->X, (kMaxK + 1) * N3)) ||
        (rc = lalloc(L, &L->Rk, kMaxK * N3)) || (rc = lalloc(L, &L->g[0], N3)) || (rc = lalloc(L, &L->g[1], N3)) ||
        (rc = lalloc(L, &L->g[2], N3)) || (rc = lalloc(L, &L->e, N3)) || (rc = lalloc(L, &L->ae, N3)) ||
        (rc = lalloc(L, &L->a2e, N3)) ||
        (rc = lalloc(L, &L->gm, n)) || (rc = lalloc(L, &L->gth, n)) || (rc = lalloc(L, &L->cr, N3)) ||
        (rc = lalloc(L, &L->cp, N3)) || (rc = lalloc(L, &L->cq, N3)) || (rc = lalloc(L, &L->part, 3 * kParts))) {
        admm_learn_destroy(L);
        return rc;
    }
    if (cudaStreamCreateWithFlags(&L->st, cudaStreamNonBlocking) != cudaSuccess) {
        admm_learn_destroy(L);
        return ADMM_ERR_CUDA;
    }
    cudaMemcpy(L->start, start, sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    if (nnz) {
        cudaMemcpy(L->col, col, sizeof(int) * nnz, cudaMemcpyHostToDevice);
        cudaMemcpy(L->val, val, sizeof(float) * nnz, cudaMemcpyHostToDevice);
    }
    cudaMemcpy(L->diag, diag, sizeof(float) * n, cudaMemcpyHostToDevice);
    if (cudaGetLastError() != cudaSuccess) {
        admm_learn_destroy(L);
        return ADMM_ERR_CUDA;
    }
    *out = L;
    return ADMM_OK;
}

void admm_learn_destroy(AdmmLearn* L) {
    if (!L) return;
    if (L->st) {
        cudaStreamSynchronize(L->st);
        cudaStreamDestroy(L->st);
    }
    for (void* p : L->allocs) cudaFree(p);
    delete L;
}

int admm_learn_loss_grad(AdmmLearn* L, int K, const float* omega, const float* beta, const float* m, const float* theta,
                         int nsamp, const float* b, const float* xc, const float* xl, const float* xs, double* loss,
                         float* g_omega, float* g_beta, float* g_m, float* g_theta) {
    if (!L || K < 1 || K > kMaxK || !omega || !beta || !m || !theta || nsamp < 1 || !b || !xc || !xl || !xs)
        return ADMM_ERR_INVALID;
    const int n = L->n;
    const size_t N3 = 3 * (size_t)n;
    const int gb = nblk(n, kT);
    cudaStream_t st = L->st;
    cudaMemcpyAsync(L->m, m, sizeof(float) * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(L->th, theta, sizeof(float) * n, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(L->gm, 0, sizeof(float) * n, st);
    cudaMemsetAsync(L->gth, 0, sizeof(float) * n, st);
    std::vector<double> go(K, 0.0), gbt(K, 0.0);
    double total = 0.0;
    int used = 0;
    for (int s = 0; s < nsamp; s++) {
        const size_t off = (size_t)s * N3;
        cudaMemcpyAsync(L->b, b + off, sizeof(float) * N3, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(L->xc, xc + off, sizeof(float) * N3, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(L->xl, xl + off, sizeof(float) * N3, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(L->xs, xs + off, sizeof(float) * N3, cudaMemcpyHostToDevice, st);
        // E_c = (xc - x*)^T A (xc - x*)
        k_t_diff<<<nblk(N3, kT), kT, 0, st>>>(L->xc, L->xs, N3, L->e);
        k_t_anorm2<<<kParts, kT, 0, st>>>(L->start, L->col, L->val, L->diag, L->e, n, L->ae, L->part);
        double Ec = 0.0;
        if (int rc = sum_parts(L, L->part, kParts, &Ec)) return rc;
        if (!(Ec > 0.0)) continue;
        used++;
        // R_c = |A (xc - x*)|^2 = |b - A xc|^2
        double Rc = 0.0;
        if (L->mu > 0.0) {
            k_t_sq<<<kParts, kT, 0, st>>>(L->ae, N3, L->part);
            if (int rc = sum_parts(L, L->part, kParts, &Rc)) return rc;
        }
        // forward
        k_t_init<<<gb, kT, 0, st>>>(L->xc, L->xl, L->th, n, L->X);
        for (int k = 0; k < K; k++) {
            const float* xk = L->X + k * N3;
            const float* xkm1 = L->X + (k > 0 ? k - 1 : 0) * N3;
            k_t_sweep<<<gb, kT, 0, st>>>(L->start, L->col, L->val, L->diag, L->m, L->b, xk, xkm1, n, omega[k],
                                         k > 0 ? beta[k] : 0.f, L->Rk + k * N3, L->X + (k + 1) * N3);
        }
        k_t_diff<<<nblk(N3, kT), kT, 0, st>>>(L->X + K * N3, L->xs, N3, L->e);
        k_t_anorm2<<<kParts, kT, 0, st>>>(L->start, L->col, L->val, L->diag, L->e, n, L->ae, L->part);
        double EK = 0.0;
        if (int rc = sum_parts(L, L->part, kParts, &EK)) return rc;
        total += EK / Ec;
        // adjoint: g_K = 2 A e_K / (E_c nsamp) (+ mu 2 A A e_K / (R_c nsamp)), in g[K % 3]
        const double sc = 2.0 / (Ec * nsamp);
        float* gK = L->g[K % 3];
        if (L->mu > 0.0 && Rc > 0.0) {
            double RK = 0.0;
            k_t_sq<<<kParts, kT, 0, st>>>(L->ae, N3, L->part);
            if (int rc = sum_parts(L, L->part, kParts, &RK)) return rc;
            total += L->mu * RK / Rc;
            k_t_anorm2<<<kParts, kT, 0, st>>>(L->start, L->col, L->val, L->diag, L->ae, n, L->a2e, L->part);
            k_t_seed<<<nblk(N3, kT), kT, 0, st>>>(gK, L->ae, L->a2e, N3, sc, L->mu * 2.0 / (Rc * nsamp));
        } else {
            k_t_seed<<<nblk(N3, kT), kT, 0, st>>>(gK, L->ae, nullptr, N3, sc, 0.0);
        }
        for (int k = K - 1; k >= 0; k--) {
            const float* g1 = L->g[(k + 1) % 3];
            const float* g2 = k + 2 <= K ? L->g[(k + 2) % 3] : nullptr;
            const float bk1 = k + 1 < K ? beta[k + 1] : 0.f;
            const float* xk = L->X + k * N3;
            const float* xkm1 = L->X + (k > 0 ? k - 1 : 0) * N3;
            k_t_adjoint<<<kParts, kT, 0, st>>>(L->start, L->col, L->val, L->diag, L->m, g1, g2, L->Rk + k * N3, xk,
                                               xkm1, n, omega[k], k > 0 ? beta[k] : 0.f, bk1, L->g[k % 3], L->gm,
                                               L->part, L->part + kParts);
            std::vector<double> h(2 * kParts);
            cudaMemcpyAsync(h.data(), L->part, sizeof(double) * 2 * kParts, cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return ADMM_ERR_CUDA;
            double so = 0.0, sb = 0.0;
            for (int i = 0; i < kParts; i++) {
                so += h[i];
                sb += h[kParts + i];
            }
            go[k] += so;
            if (k > 0) gbt[k] += sb;
        }
        k_t_theta<<<gb, kT, 0, st>>>(L->g[0], L->xc, L->xl, n, L->gth);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ADMM_ERR_CUDA;
    if (loss) *loss = used ? total / nsamp : 0.0;
    if (g_omega)
        for (int k = 0; k < K; k++) g_omega[k] = (float)go[k];
    if (g_beta)
        for (int k = 0; k < K; k++) g_beta[k] = (float)gbt[k];
    if (g_m && cudaMemcpy(g_m, L->gm, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return ADMM_ERR_CUDA;
    if (g_theta && cudaMemcpy(g_theta, L->gth, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return ADMM_ERR_CUDA;
    return ADMM_OK;
}

int admm_learn_set_residual_weight(AdmmLearn* L, double mu) {
    if (!L || !(mu >= 0.0) || !std::isfinite(mu)) return ADMM_ERR_INVALID;
    L->mu = mu;
    return ADMM_OK;
}

int admm_learn_solve(AdmmLearn* L, const float* b, float* x, double rel_tol, int max_iter, int* iters) {
    if (!L || !b || !x || max_iter < 0) return ADMM_ERR_INVALID;
    const int n = L->n;
    const size_t N3 = 3 * (size_t)n;
    cudaStream_t st = L->st;
    cudaMemcpyAsync(L->b, b, sizeof(float) * N3, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(L->xs, x, sizeof(float) * N3, cudaMemcpyHostToDevice, st);
    k_cg_init<<<kParts, kT, 0, st>>>(L->start, L->col, L->val, L->diag, L->b, L->xs, n, L->cr, L->cp, L->part);
    double rz = 0.0;
    if (int rc = sum_parts(L, L->part, kParts, &rz)) return rc;
    const double rz0 = rz;
    int it = 0;
    for (; it < max_iter && rz > rel_tol * rel_tol * rz0 && rz > 0.0; it++) {
        k_cg_q<<<kParts, kT, 0, st>>>(L->start, L->col, L->val, L->diag, L->cp, n, L->cq, L->part);
        double pq = 0.0;
        if (int rc = sum_parts(L, L->part, kParts, &pq)) return rc;
        if (!(pq > 0.0)) break;
        const double alpha = rz / pq;
        k_cg_xr<<<kParts, kT, 0, st>>>(L->diag, L->cp, L->cq, n, alpha, L->xs, L->cr, L->part);
        double rzn = 0.0;
        if (int rc = sum_parts(L, L->part, kParts, &rzn)) return rc;
        k_cg_p<<<nblk(n, kT), kT, 0, st>>>(L->diag, L->cr, n, rzn / rz, L->cp);
        rz = rzn;
    }
    if (cudaMemcpy(x, L->xs, sizeof(float) * N3, cudaMemcpyDeviceToHost) != cudaSuccess) return ADMM_ERR_CUDA;
    if (iters) *iters = it;
    return cudaGetLastError() == cudaSuccess ? ADMM_OK : ADMM_ERR_CUDA;
}

}  // extern "C"
