// ref_pin_solver.cpp -- TEST INFRASTRUCTURE ONLY.  Runs the reference's own contact
// and Jacobi kernels on the host to pin the oracle's restatements of them:
// compute_Scc_kernel, update_p_kernel, get_delta_u_kernel and update_p
// (src/solver/contact_solver.cu) and JacobiFunctor (src/solver/jacobi_solver.cu).
// oracle/ref_extract.py cuts those definitions out of the reference tree into
// oracle/_ref/solver_extract.inc at build time (see oracle/Makefile); nothing of them
// is copied into this repository.  Each kernel runs serially, one "thread" per index,
// so its atomics are plain read-modify-writes in index order.  Output: oracle/_ref/.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "cuda.h"

struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int4 { int x, y, z, w; };
static inline float3 make_float3(float a, float b, float c) { return float3{a, b, c}; }
struct PinDim3 { unsigned x = 0, y = 0, z = 0; };
static PinDim3 threadIdx, blockIdx, blockDim;
#define __global__ static
static inline int atomicAdd(int* a, int v) { const int o = *a; *a += v; return o; }
static inline float atomicAdd(float* a, float v) { const float o = *a; *a += v; return o; }

#include "dist_g.cuh"  // Result<T>, named in compute_Scc_kernel's signature

namespace ADU { using Real = float; }
using namespace ADU;

#include "solver_extract.inc"

namespace {
// One launch of n "threads" (blockDim n, one block), run in index order.
template <class F>
void serial(int n, F f) {
    blockDim.x = (unsigned)(n > 0 ? n : 1);
    blockIdx.x = 0;
    for (int i = 0; i < n; i++) {
        threadIdx.x = (unsigned)i;
        f();
    }
}
}  // namespace

extern "C" {

// compute_Scc_kernel over nc contacts: v4 [nc x 4], bary4 [nc x 4], start/count per vertex
// (the CSR of the per-vertex contact lists), w / w_inv per vertex, h_cN [nc], normal3
// [nc x 3]; out Gamma_c [nc x 4], K_c [nc x 3], and the lists (involved contact, Gamma_i).
void ref_scc_f(int nc, const int* v4, const float* bary4, const int* start, const int* cnt, const float* w,
               const float* winv, const float* hcn, const float* normal3, float gamma, float eps, float dt_inv,
               int nv, float* Gam4, float* Kc3, int* involved, float* gamma_i) {
    int* fill = new int[nv > 0 ? nv : 1]();
    float3* du = new float3[nc > 0 ? nc : 1]();
    serial(nc, [&] {
        compute_Scc_kernel(reinterpret_cast<const int4*>(v4), nullptr, start, reinterpret_cast<const float4*>(bary4),
                           cnt, w, winv, hcn, reinterpret_cast<const float3*>(normal3), gamma, eps, nc, dt_inv, fill,
                           involved, gamma_i, reinterpret_cast<float4*>(Gam4), reinterpret_cast<float3*>(Kc3), du);
    });
    delete[] fill;
    delete[] du;
}

// update_p_kernel: p += Gamma_c r_c on the dynamic vertices (index < n_dyn).
void ref_warm_p_f(int nc, const int* v4, const float* Gam4, float* p, const float* rc3, int n_dyn) {
    serial(nc, [&] {
        update_p_kernel(nc, reinterpret_cast<const int4*>(v4), reinterpret_cast<const float4*>(Gam4), p,
                        reinterpret_cast<float3*>(const_cast<float*>(rc3)), n_dyn);
    });
}

// get_delta_u_kernel with one friction coefficient: du3 out, rc3 updated.
void ref_delta_u_f(int nc, float mu, const int* v4, const float* bary4, const float* p, const float* Kc3,
                   const float* normal3, float* du3, float* rc3) {
    serial(nc, [&] {
        get_delta_u_kernel(nc, mu, reinterpret_cast<const int4*>(v4), reinterpret_cast<const float4*>(bary4), p,
                           reinterpret_cast<const float3*>(Kc3), reinterpret_cast<const float3*>(normal3),
                           reinterpret_cast<float3*>(du3), reinterpret_cast<float3*>(rc3));
    });
}

// update_p: p[v] += sum over v's list of du[contact] Gamma_i.
void ref_gather_p_f(int nv, const int* involved, const int* start, const float* gamma_i, const float* du3, float* p) {
    serial(nv, [&] { update_p(nv, involved, start, gamma_i, reinterpret_cast<const float3*>(du3), p); });
}

// One Jacobi sweep over CSR rows with JacobiFunctor.
void ref_jacobi_sweep_f(int rows, const int* start, const int* col, const float* val, const float* diag,
                        const float* b, const float* x, float* xn) {
    JacobiFunctor f(diag, val, col, start, b, x, xn, rows);
    for (int i = 0; i < rows; i++) f(i);
}

}  // extern "C"
