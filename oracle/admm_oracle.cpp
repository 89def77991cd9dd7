// admm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A CPU restatement of the reference's GPU ADMM substep (ADMMImplGPU::step,
// src/solver/backend_gpu/admm_impl_gpu.cu:256-344), templated on the real type
// so it runs in FP64 (the accuracy reference) and FP32 (the reference's own
// ADU::Real, src/mutils/common_types.h:10).  It is the checker of the CUDA
// library in tests/, __graft_entry__.smoke() and the CPU-baseline leg of
// bench.py; the product never calls it.  Built with -ffp-contract=off.
//
// Parity status: the narrow-phase predicates and the SVD-based prox are pinned
// against the reference's own dist_g.cuh / svd_fast3.cuh compiled on the host
// (oracle/ref_pin.cpp); everything else is a restatement of the cited lines
// ("parity unpinned": the reference ships no tests, fixtures or golden vectors
// and cannot be built here).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/admm_b200.h"
#include <cstdio>

#include "oracle_math.hpp"

using namespace orc;

namespace {

struct Csr {
    std::vector<int> start, col;
    std::vector<double> val;
};

struct Contact {
    int v[4];
    int type;  // 0 edge-edge, 1 point-triangle (contact_solver.cu:136)
    float bary_raw[3];
    double bary[4];
    double normal[3];
    double point[3];
    double gap;  // h_cN - thickness
};

// ---------------------------------------------------------------------------
// DCD: leaf-overlap filter (lbvh.cu:43-49) + region-0 narrow phase, evaluated in
// float with the reference's operation order.  The pair set does not depend on
// the tree: an internal node's box contains its leaves' boxes and the overlap
// test is monotone, so a pair is reported iff its leaf boxes pass the test and
// the predicate accepts it.  A uniform grid replaces the tree on the CPU.
// ---------------------------------------------------------------------------
struct Grid {
    float org[3];
    float cell;
    int dims[3];
    std::unordered_map<int64_t, std::vector<int>> cells;
    std::vector<int> big;  // boxes spanning too many cells: tested against every query
    int64_t key(int i, int j, int k) const { return (int64_t(i) * dims[1] + j) * dims[2] + k; }
    void range(const Box<float>& b, float pad, int lo[3], int hi[3]) const {
        const float* l = &b.lo.x;
        const float* u = &b.up.x;
        for (int a = 0; a < 3; a++) {
            lo[a] = std::max(0, std::min(dims[a] - 1, int(std::floor((l[a] - pad - org[a]) / cell))));
            hi[a] = std::max(0, std::min(dims[a] - 1, int(std::floor((u[a] + pad - org[a]) / cell))));
        }
    }
};

static Box<float> box_of(const float* x, const int* ids, int n) {
    Box<float> b;
    b.lo = mk(1e32f, 1e32f, 1e32f);
    b.up = mk(-1e32f, -1e32f, -1e32f);
    for (int i = 0; i < n; i++) {
        const float* p = x + 3 * ids[i];
        b.lo.x = std::min(b.lo.x, p[0]); b.lo.y = std::min(b.lo.y, p[1]); b.lo.z = std::min(b.lo.z, p[2]);
        b.up.x = std::max(b.up.x, p[0]); b.up.y = std::max(b.up.y, p[1]); b.up.z = std::max(b.up.z, p[2]);
    }
    return b;
}

static void build_grid(Grid& g, const std::vector<Box<float>>& boxes, float gap) {
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    std::vector<float> ext(boxes.size());
    for (size_t i = 0; i < boxes.size(); i++) {
        const Box<float>& b = boxes[i];
        lo[0] = std::min(lo[0], b.lo.x); lo[1] = std::min(lo[1], b.lo.y); lo[2] = std::min(lo[2], b.lo.z);
        hi[0] = std::max(hi[0], b.up.x); hi[1] = std::max(hi[1], b.up.y); hi[2] = std::max(hi[2], b.up.z);
        ext[i] = std::max(b.up.x - b.lo.x, std::max(b.up.y - b.lo.y, b.up.z - b.lo.z));
    }
    float span = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    float e90 = 0.f;
    if (!ext.empty()) {
        std::vector<float> e = ext;
        size_t k = (e.size() * 9) / 10;
        std::nth_element(e.begin(), e.begin() + k, e.end());
        e90 = e[k];
    }
    g.cell = std::max(e90 + 2.f * gap, span / 1024.f);
    if (!(g.cell > 0.f)) g.cell = 1.f;
    for (int a = 0; a < 3; a++) {
        g.org[a] = lo[a] - 2.f * gap - g.cell;
        g.dims[a] = std::max(1, int((hi[a] - g.org[a] + 2.f * gap) / g.cell) + 2);
    }
    for (int i = 0; i < (int)boxes.size(); i++) {
        int l[3], h[3];
        g.range(boxes[i], 0.f, l, h);
        const int64_t ncell = int64_t(h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1);
        if (ncell > 64) { g.big.push_back(i); continue; }
        for (int a = l[0]; a <= h[0]; a++)
            for (int b = l[1]; b <= h[1]; b++)
                for (int c = l[2]; c <= h[2]; c++) g.cells[g.key(a, b, c)].push_back(i);
    }
}

struct RawPair {
    int v[4];
    Result<float> r;
};

// All DCD pairs on float positions x (n x 3).  VF: each surface vertex against
// every surface triangle not containing it (lbvh.cu:1693-1748).  EE: each edge
// against every edge with a larger index sharing no vertex (lbvh.cu:1750-1813).
// semantics 0: the GPU backend's predicates (region 0, 0 <= d < thickness,
// boxes within the gap).  semantics 1: the CPU backend's ProximalQuery
// (narrow_phase.cpp:192-469): no pair of two static elements (first vertex of
// each at or above static_begin), point-triangle at any closest point with
// d <= thickness, edge-edge with d < thickness unless both closest points are
// segment end points; the box test is only a candidate filter there, so the
// candidates are every element of the cells within the gap.
static void dcd_all(const float* x, const std::vector<int>& sv, const std::vector<int>& st,
                    const std::vector<int>& se, float thickness, std::vector<RawPair>& out,
                    int semantics = 0, int static_begin = 1 << 30) {
    const int nsv = (int)sv.size(), nst = (int)st.size() / 3, nse = (int)se.size() / 2;
    std::vector<Box<float>> tb(nst), eb(nse);
    for (int i = 0; i < nst; i++) tb[i] = box_of(x, &st[3 * i], 3);
    for (int i = 0; i < nse; i++) eb[i] = box_of(x, &se[2 * i], 2);
    out.clear();
    auto P = [&](int i) { return mk(x[3 * i], x[3 * i + 1], x[3 * i + 2]); };
    if (nst > 0) {
        Grid g;
        build_grid(g, tb, thickness);
        std::vector<std::vector<RawPair>> local(nsv);
#pragma omp parallel for schedule(dynamic, 64)
        for (int q = 0; q < nsv; q++) {
            int v = sv[q];
            Box<float> qb;
            qb.lo = qb.up = P(v);
            int l[3], h[3];
            g.range(qb, thickness * 1.01f + 1e-6f, l, h);
            std::vector<int> cand;
            for (int a = l[0]; a <= h[0]; a++)
                for (int b = l[1]; b <= h[1]; b++)
                    for (int c = l[2]; c <= h[2]; c++) {
                        auto it = g.cells.find(g.key(a, b, c));
                        if (it != g.cells.end()) cand.insert(cand.end(), it->second.begin(), it->second.end());
                    }
            cand.insert(cand.end(), g.big.begin(), g.big.end());
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            for (int f : cand) {
                const int* t = &st[3 * f];
                if (v == t[0] || v == t[1] || v == t[2]) continue;
                if (semantics == 1) {
                    if (v >= static_begin && t[0] >= static_begin) continue;
                    Result<float> r = gt_point_triangle(P(v), P(t[0]), P(t[1]), P(t[2]));
                    if (r.distance <= thickness) local[q].push_back(RawPair{{v, t[0], t[1], t[2]}, r});
                    continue;
                }
                if (!overlap(qb, tb[f], thickness)) continue;
                Result<float> r = dcd_pt(P(v), P(t[0]), P(t[1]), P(t[2]));
                if (r.distance < thickness && r.distance >= 0.f) local[q].push_back(RawPair{{v, t[0], t[1], t[2]}, r});
            }
        }
        for (auto& l : local) out.insert(out.end(), l.begin(), l.end());
    }
    if (nse > 0) {
        Grid g;
        build_grid(g, eb, thickness);
        std::vector<std::vector<RawPair>> local(nse);
#pragma omp parallel for schedule(dynamic, 64)
        for (int e = 0; e < nse; e++) {
            int l[3], h[3];
            g.range(eb[e], thickness * 1.01f + 1e-6f, l, h);
            std::vector<int> cand;
            for (int a = l[0]; a <= h[0]; a++)
                for (int b = l[1]; b <= h[1]; b++)
                    for (int c = l[2]; c <= h[2]; c++) {
                        auto it = g.cells.find(g.key(a, b, c));
                        if (it != g.cells.end()) cand.insert(cand.end(), it->second.begin(), it->second.end());
                    }
            cand.insert(cand.end(), g.big.begin(), g.big.end());
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            const int ea = se[2 * e], eb_ = se[2 * e + 1];
            for (int o : cand) {
                if (o <= e) continue;
                const int oa = se[2 * o], ob = se[2 * o + 1];
                if (ea == oa || ea == ob || eb_ == oa || eb_ == ob) continue;
                if (semantics == 1) {
                    if (ea >= static_begin && oa >= static_begin) continue;
                    Result<float> r = gt_segment_segment(P(ea), P(eb_), P(oa), P(ob));
                    const bool corner = (r.bary[0] == 0.f || r.bary[0] == 1.f) && (r.bary[1] == 0.f || r.bary[1] == 1.f);
                    if (r.distance < thickness && !corner) local[e].push_back(RawPair{{ea, eb_, oa, ob}, r});
                    continue;
                }
                if (!overlap(eb[e], eb[o], thickness)) continue;
                Result<float> r = dcd_ee(P(ea), P(eb_), P(oa), P(ob));
                if (r.distance < thickness && r.distance >= 0.f) local[e].push_back(RawPair{{ea, eb_, oa, ob}, r});
            }
        }
        for (auto& l : local) out.insert(out.end(), l.begin(), l.end());
    }
}

// ---------------------------------------------------------------------------
// Exact solve of the CPU backend's damped system (SimplicialLLT of m_A_damp,
// admm_impl_cpu.cpp:248-250, solved per column, linear_solver_cpu.h:16-23):
// FP64 envelope (skyline) Cholesky A = L L^T after a reverse Cuthill-McKee
// ordering of the symmetric pattern.  The envelope of row i spans its first
// non-zero column to the diagonal; Cholesky creates no fill outside it.
// ---------------------------------------------------------------------------
struct EnvelopeCholesky {
    int n = 0;
    std::vector<int> perm, iperm;  // new -> old, old -> new
    std::vector<int> first;        // first column of row i's envelope (new order)
    std::vector<long> off;         // start of row i in L (entries first[i] .. i)
    std::vector<double> L;

    // Reverse Cuthill-McKee over every connected component, each started from a
    // pseudo-peripheral vertex (two breadth-first passes from a vertex of least degree).
    void order(const std::vector<int>& start, const std::vector<int>& col) {
        std::vector<int> deg(n);
        for (int i = 0; i < n; i++) deg[i] = start[i + 1] - start[i];
        std::vector<char> seen(n, 0);
        std::vector<int> out;
        out.reserve(n);
        auto bfs = [&](int root, std::vector<int>& lev, std::vector<char>& mark) {
            lev.clear();
            lev.push_back(root);
            mark[root] = 1;
            for (size_t h = 0; h < lev.size(); h++) {
                const int u = lev[h];
                std::vector<int> nb;
                for (int a = start[u]; a < start[u + 1]; a++)
                    if (!mark[col[a]]) { mark[col[a]] = 1; nb.push_back(col[a]); }
                std::sort(nb.begin(), nb.end(), [&](int x, int y) { return deg[x] != deg[y] ? deg[x] < deg[y] : x < y; });
                lev.insert(lev.end(), nb.begin(), nb.end());
            }
        };
        std::vector<int> comp;
        for (int s0 = 0; s0 < n; s0++) {
            if (seen[s0]) continue;
            std::vector<char> mark(seen);
            bfs(s0, comp, mark);
            int root = s0;
            for (int v : comp) if (deg[v] < deg[root]) root = v;
            mark = seen;
            bfs(root, comp, mark);
            root = comp.back();
            mark = seen;
            bfs(root, comp, mark);
            for (int v : comp) seen[v] = 1;
            out.insert(out.end(), comp.rbegin(), comp.rend());
        }
        perm = out;
        iperm.assign(n, 0);
        for (int i = 0; i < n; i++) iperm[perm[i]] = i;
    }

    // A: off-diagonal CSR (symmetric pattern) and diagonal.
    bool factor(int nn, const std::vector<int>& start, const std::vector<int>& col, const std::vector<double>& val,
                const std::vector<double>& diag) {
        n = nn;
        order(start, col);
        first.assign(n, 0);
        for (int i = 0; i < n; i++) {
            int f = i;
            const int o = perm[i];
            for (int a = start[o]; a < start[o + 1]; a++) f = std::min(f, iperm[col[a]]);
            first[i] = f;
        }
        off.assign(n + 1, 0);
        for (int i = 0; i < n; i++) off[i + 1] = off[i] + (i - first[i] + 1);
        L.assign(off[n], 0.0);
        for (int i = 0; i < n; i++) {
            const int o = perm[i];
            L[off[i] + (i - first[i])] = diag[o];
            for (int a = start[o]; a < start[o + 1]; a++) {
                const int j = iperm[col[a]];
                if (j < i) L[off[i] + (j - first[i])] += val[a];
            }
        }
        for (int i = 0; i < n; i++) {
            double* Li = &L[off[i]];
            for (int j = first[i]; j < i; j++) {
                const double* Lj = &L[off[j]];
                const int k0 = std::max(first[i], first[j]);
                double s = Li[j - first[i]];
                for (int k = k0; k < j; k++) s -= Li[k - first[i]] * Lj[k - first[j]];
                Li[j - first[i]] = s / Lj[j - first[j]];
            }
            double s = Li[i - first[i]];
            for (int k = first[i]; k < i; k++) s -= Li[k - first[i]] * Li[k - first[i]];
            if (!(s > 0.0)) return false;
            Li[i - first[i]] = std::sqrt(s);
        }
        return true;
    }

    // x = A^-1 b for one column (original order).
    void solve(const double* b, double* x) const {
        std::vector<double> y(n);
        for (int i = 0; i < n; i++) y[i] = b[perm[i]];
        for (int i = 0; i < n; i++) {
            const double* Li = &L[off[i]];
            double s = y[i];
            for (int k = first[i]; k < i; k++) s -= Li[k - first[i]] * y[k];
            y[i] = s / Li[i - first[i]];
        }
        for (int i = n - 1; i >= 0; i--) {
            const double* Li = &L[off[i]];
            y[i] /= Li[i - first[i]];
            for (int k = first[i]; k < i; k++) y[k] -= Li[k - first[i]] * y[i];
        }
        for (int i = 0; i < n; i++) x[perm[i]] = y[i];
    }
};

// ---------------------------------------------------------------------------
// The ADMM oracle.
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Per-contact and per-row pieces of the GPU backend's contact and global steps, shared by
// the Oracle below and by the orc_*_f entry points that pin them to the reference's own
// kernels (tests/test_oracle_golden.py).
// ---------------------------------------------------------------------------

// S_c, Gamma_c and K_c of one contact (compute_Scc_kernel, contact_solver.cu:188-232):
// S_c = eps + sum_k bary_k^2 w_inv[v_k] n[v_k], Gamma_k = bary_k / (S_c w[v_k]),
// K_c = dt_inv h_cN normal gamma.  cpu_backend: the CPU backend's form (compute_Scc,
// admm_impl_cpu.cpp:361-380): no per-vertex counts, Gamma of static vertices (w > 1e7) zero.
template <class R>
static void scc_contact(const Contact& ct, const int* cnt, const R* w, const R* winv, R eps, R gam, R dt_inv,
                        bool cpu_backend, R* Gam4, R* Kc3) {
    R t[4];
    for (int k = 0; k < 4; k++)
        t[k] = (R)ct.bary[k] * (R)ct.bary[k] * winv[ct.v[k]] * (cpu_backend ? R(1) : (R)cnt[ct.v[k]]);
    const R Sc = eps + (((t[0] + t[1]) + t[2]) + t[3]);
    for (int k = 0; k < 4; k++) {
        Gam4[k] = (R)ct.bary[k] / (Sc * w[ct.v[k]]);
        if (cpu_backend && w[ct.v[k]] > R(1e7)) Gam4[k] = 0;
    }
    for (int k = 0; k < 3; k++) Kc3[k] = dt_inv * (R)ct.gap * (R)ct.normal[k] * gam;
}

// One friction-cone projection of a contact (get_delta_u_kernel, contact_solver.cu:337-379):
// u = sum_k bary_k p[v_k] + K_c, u* = u - r_c split along the normal; a compressive u*
// loses its normal part and its tangential part is scaled onto the cone of slope mu;
// du = u*_new - u, r_c += du.
template <class R>
static void cone_step(const Contact& ct, R mu, const R* p, const R* Kc3, R* rc3, R* du3) {
    R u[3];
    for (int a = 0; a < 3; a++)
        u[a] = (((R)ct.bary[0] * p[3 * ct.v[0] + a] + (R)ct.bary[1] * p[3 * ct.v[1] + a]) +
                (R)ct.bary[2] * p[3 * ct.v[2] + a]) + (R)ct.bary[3] * p[3 * ct.v[3] + a] + Kc3[a];
    R nrm[3] = {(R)ct.normal[0], (R)ct.normal[1], (R)ct.normal[2]};
    R us[3];
    for (int a = 0; a < 3; a++) us[a] = u[a] - rc3[a];
    R uN = (nrm[0] * us[0] + nrm[1] * us[1]) + nrm[2] * us[2];
    R uT[3];
    for (int a = 0; a < 3; a++) uT[a] = us[a] - uN * nrm[a];
    if (uN < 0) {
        R tau = std::sqrt((uT[0] * uT[0] + uT[1] * uT[1]) + uT[2] * uT[2]);
        R alpha = -mu * uN;
        uN = 0;
        if (tau <= alpha) uT[0] = uT[1] = uT[2] = 0;
        else { R sc = R(1) - alpha / tau; for (int a = 0; a < 3; a++) uT[a] = sc * uT[a]; }
    }
    for (int a = 0; a < 3; a++) {
        R un = uN * nrm[a] + uT[a];
        du3[a] = un - u[a];
        rc3[a] = rc3[a] + du3[a];
    }
}

// p[v] += sum over v's contact slots of du_c Gamma_{c,k}, slots in list order
// (update_p, contact_solver.cu:381-399); list entries are 4 c + k.
template <class R>
static void gather_p(int nv, const int* vstart, const int* vlist, const R* Gam, const R* du, R* p) {
    for (int vi = 0; vi < nv; vi++) {
        R d[3] = {0, 0, 0};
        for (int s = vstart[vi]; s < vstart[vi + 1]; s++) {
            int e = vlist[s];
            int c = e >> 2, k = e & 3;
            for (int a = 0; a < 3; a++) d[a] = d[a] + du[3 * c + a] * Gam[4 * c + k];
        }
        for (int a = 0; a < 3; a++) p[3 * vi + a] += d[a];
    }
}

// One Jacobi sweep xn = D^-1 (b - (A - D) x) over CSR rows (JacobiFunctor,
// jacobi_solver.cu:52-98), off-diagonal products summed in column order.
template <class R, class V>
static void jacobi_sweep(int rows, const int* start, const int* col, const V* val, const R* diag, const R* b,
                         const R* x, R* xn) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < rows; i++) {
        R acc[3] = {0, 0, 0};
        for (int a = start[i]; a < start[i + 1]; a++) {
            int j = col[a];
            for (int k = 0; k < 3; k++) acc[k] += x[3 * j + k] * (R)val[a];
        }
        for (int k = 0; k < 3; k++) xn[3 * i + k] = (b[3 * i + k] - acc[k]) / diag[i];
    }
}

template <class R>
struct Oracle {
    // scene
    int n = 0, nd = 0, m = 0;
    std::vector<R> mass;
    std::vector<int> fixed;
    int ntri = 0, ntet = 0, nbend = 0, npin = 0;
    int tri_sr = 0, tet_sr = 0, bend_sr = 0, pin_sr = 0;
    std::vector<int> tri_inds, tet_inds, bend_off, bend_inds, pin_inds;
    std::vector<R> tri_binv, tet_binv, bend_coef, bend_rest, pin_pos;
    std::vector<R> wrow;  // w per row
    std::vector<int> surf_tris, surf_edges, surf_verts;
    std::vector<R> cw, cwinv;
    std::vector<char> is_surf;
    R dt, g, mu, kappa, beta;
    std::vector<R> vmu;  // per-vertex friction (empty: mu everywhere)
    std::vector<R> cmu;  // per contact: the coefficient of its first dynamic vertex
    float thickness;
    int semantics = 0;  // contact predicates: 0 GPU backend, 1 CPU backend
    int admm_max_iter, dcd_interval, gs_max_iter, jacobi_iter;
    bool contact, ws_ue, ws_uc;
    float residual_tol = 0.f;
    int chunk = 0;
    int global_solver = 0, pcg_iter = 0;
    std::vector<R> pblock;  // [9 nd] learned 3x3 preconditioner blocks (global_solver 2)
    // semantics of the reference's CPU backend (backend_semantics 1)
    int backend = 0;
    double damp_k_L = 0.0, damp_k_M = 0.0;
    Csr Damp;                    // off-diagonal part of the damping matrix (added to A too)
    std::vector<double> Ddiag;   // its diagonal
    EnvelopeCholesky chol;       // exact factor of the damped A
    // learned global step (global_solver 3): sweeps, coefficients, per-vertex m and theta
    int learn_K = 0;
    std::vector<R> learn_omega, learn_beta, learn_m, learn_theta, xl;
    bool warm_on = true;  // the warm start is still on in this substep (adaptive restart)
    long long learn_substeps = 0, learn_fallbacks = 0, learn_solves = 0, learn_failed = 0;
    // matrices
    Csr D;        // m x nd
    Csr A;        // nd x nd off-diagonal part
    std::vector<R> Adiag;
    Csr DtW2;     // nd x m, h^2 D^T W^2
    std::vector<R> dt2Wc;  // nd
    // state (row-major x3)
    std::vector<R> x0_init, v0_init;
    std::vector<R> x0, v, x, p, mxt, b, Ue, Uc, z;
    // contacts
    std::vector<Contact> cts;
    std::vector<R> Gam;  // 4 per contact
    std::vector<R> Kc, rc, du;
    std::vector<int> vstart, vlist;  // vertex -> (contact*4 + slot)
    int peak = 0;
    // residuals of the last iteration
    double last_primal = 0, last_dual = 0;
    std::vector<R> xprev;

    void setup(const AdmmB200Desc* d) {
        n = d->n_vert; nd = d->n_dyn; m = d->n_rows;
        mass.assign(d->mass, d->mass + n);
        fixed.assign(n, 0);
        if (d->is_fixed) fixed.assign(d->is_fixed, d->is_fixed + n);
        ntri = d->n_tri; ntet = d->n_tet; nbend = d->n_bend; npin = d->n_pin;
        tri_sr = d->tri_start_row; tet_sr = d->tet_start_row; bend_sr = d->bend_start_row; pin_sr = d->pin_start_row;
        tri_inds.assign(d->tri_inds, d->tri_inds + 3 * ntri);
        tri_binv.assign(d->tri_binv, d->tri_binv + 4 * ntri);
        tet_inds.assign(d->tet_inds, d->tet_inds + 4 * ntet);
        tet_binv.assign(d->tet_binv, d->tet_binv + 9 * ntet);
        bend_off.assign(d->bend_offsets, d->bend_offsets + nbend + 1);
        int nbe = nbend ? bend_off[nbend] : 0;
        bend_inds.assign(d->bend_inds, d->bend_inds + nbe);
        bend_coef.assign(d->bend_coeffs, d->bend_coeffs + nbe);
        bend_rest.assign(nbend, R(0));
        if (d->bend_rest_norm) bend_rest.assign(d->bend_rest_norm, d->bend_rest_norm + nbend);
        pin_inds.assign(d->pin_inds, d->pin_inds + npin);
        pin_pos.assign(d->pin_pos, d->pin_pos + 3 * npin);
        wrow.assign(m, R(0));
        for (int c = 0; c < ntri; c++) for (int r = 0; r < 2; r++) wrow[tri_sr + 2 * c + r] = d->tri_w[c];
        for (int c = 0; c < ntet; c++) for (int r = 0; r < 3; r++) wrow[tet_sr + 3 * c + r] = d->tet_w[c];
        for (int c = 0; c < nbend; c++) wrow[bend_sr + c] = d->bend_w[c];
        for (int c = 0; c < npin; c++) wrow[pin_sr + c] = d->pin_w[c];
        surf_tris.assign(d->surf_tris, d->surf_tris + 3 * d->n_surf_tri);
        surf_edges.assign(d->surf_edges, d->surf_edges + 2 * d->n_surf_edge);
        surf_verts.assign(d->surf_verts, d->surf_verts + d->n_surf_vert);
        cw.assign(d->contact_w, d->contact_w + n);
        cwinv.assign(n, R(0));
        for (int i = 0; i < nd; i++) cwinv[i] = R(1) / cw[i];  // solver_config_applier.cpp:45
        is_surf.assign(n, 0);
        for (int s : surf_verts) is_surf[s] = 1;
        dt = d->dt; g = d->g; mu = d->mu; kappa = d->kappa; beta = d->beta; thickness = d->thickness;
        semantics = d->contact_semantics;
        backend = d->backend_semantics;
        if (backend == 1) semantics = 1;
        damp_k_L = d->damp_k_L;
        damp_k_M = d->damp_k_M;
        if (d->vert_mu) vmu.assign(d->vert_mu, d->vert_mu + d->n_vert);
        admm_max_iter = d->admm_max_iter; dcd_interval = std::max(1, d->dcd_interval);
        gs_max_iter = d->gs_max_iter; jacobi_iter = d->jacobi_iter;
        contact = d->enable_contact != 0; ws_ue = d->warmstart_ue != 0; ws_uc = d->warmstart_uc != 0;
        residual_tol = d->residual_tol;
        global_solver = d->global_solver;
        pcg_iter = d->pcg_iter > 0 ? d->pcg_iter : std::max(1, d->jacobi_iter / 2);
        {
            const int every = d->residual_check_every > 0 ? d->residual_check_every : dcd_interval;
            chunk = (every + dcd_interval - 1) / dcd_interval * dcd_interval;
        }
        x0_init.assign(3 * n, R(0));
        v0_init.assign(3 * n, R(0));
        for (int i = 0; i < 3 * n; i++) x0_init[i] = d->x0[i];
        if (d->v0) for (int i = 0; i < 3 * n; i++) v0_init[i] = d->v0[i];
        precompute();
        reset();
    }

    // D rows (Constraint::get_D): tri G = S*Binv (triangle_constraint.h:64-95),
    // tet G = S*Binv (tetrahedral_constraint.h:58-89), bending coeffs
    // (bending_constraint.h:173-193), pin 1 (pin_constraint.h:37-48).
    void precompute() {
        std::vector<std::vector<std::pair<int, R>>> rows(m);
        for (int c = 0; c < ntri; c++) {
            const R* B = &tri_binv[4 * c];  // row-major 2x2
            R G[3][2];
            for (int r = 0; r < 2; r++) {
                G[0][r] = -(B[0 * 2 + r] + B[1 * 2 + r]);
                G[1][r] = B[0 * 2 + r];
                G[2][r] = B[1 * 2 + r];
            }
            for (int r = 0; r < 2; r++)
                for (int j = 0; j < 3; j++) rows[tri_sr + 2 * c + r].push_back({tri_inds[3 * c + j], G[j][r]});
        }
        for (int c = 0; c < ntet; c++) {
            const R* B = &tet_binv[9 * c];
            R G[4][3];
            for (int r = 0; r < 3; r++) {
                G[0][r] = -((B[0 * 3 + r] + B[1 * 3 + r]) + B[2 * 3 + r]);
                G[1][r] = B[0 * 3 + r];
                G[2][r] = B[1 * 3 + r];
                G[3][r] = B[2 * 3 + r];
            }
            for (int r = 0; r < 3; r++)
                for (int j = 0; j < 4; j++) rows[tet_sr + 3 * c + r].push_back({tet_inds[4 * c + j], G[j][r]});
        }
        for (int c = 0; c < nbend; c++)
            for (int k = bend_off[c]; k < bend_off[c + 1]; k++) rows[bend_sr + c].push_back({bend_inds[k], bend_coef[k]});
        for (int c = 0; c < npin; c++) rows[pin_sr + c].push_back({pin_inds[c], R(1)});
        // CSR of D with duplicates summed and columns sorted (Eigen setFromTriplets)
        D.start.assign(m + 1, 0);
        D.col.clear(); D.val.clear();
        for (int r = 0; r < m; r++) {
            auto& e = rows[r];
            std::sort(e.begin(), e.end(), [](auto& a, auto& b) { return a.first < b.first; });
            for (size_t i = 0; i < e.size(); i++) {
                if (!D.col.empty() && (int)D.start[r] < (int)D.col.size() && D.col.back() == e[i].first) {
                    D.val.back() += (double)e[i].second;
                } else {
                    D.col.push_back(e[i].first);
                    D.val.push_back((double)e[i].second);
                }
            }
            D.start[r + 1] = (int)D.col.size();
        }
        const R h2 = dt * dt;
        // A = M + h^2 D^T W^2 D + h^2 W_c  (admm_impl_gpu.cu:164-234)
        std::vector<std::unordered_map<int, double>> arow(nd);
        std::vector<std::vector<std::pair<int, double>>> dtw(nd);
        for (int r = 0; r < m; r++) {
            double w2 = (double)wrow[r] * (double)wrow[r] * (double)h2;
            for (int a = D.start[r]; a < D.start[r + 1]; a++) {
                int i = D.col[a];
                dtw[i].push_back({r, w2 * D.val[a]});
                for (int bb = D.start[r]; bb < D.start[r + 1]; bb++) arow[i][D.col[bb]] += w2 * D.val[a] * D.val[bb];
            }
        }
        // the CPU backend's damping (admm_impl_cpu.cpp:181-191, 221): Damp = dt (damp_k_L
        // Dd^T Wd Dd + damp_k_M M) over the triangle, tet and bending rows, Wd = diag(w);
        // A_damp = A + Damp
        if (backend == 1) {
            std::vector<std::unordered_map<int, double>> drow(nd);
            auto damped = [&](int r) {
                return (ntri && r >= tri_sr && r < tri_sr + 2 * ntri) || (ntet && r >= tet_sr && r < tet_sr + 3 * ntet) ||
                       (nbend && r >= bend_sr && r < bend_sr + nbend);
            };
            for (int r = 0; r < m; r++) {
                if (!damped(r)) continue;
                const double sw = (double)dt * damp_k_L * (double)wrow[r];
                for (int a = D.start[r]; a < D.start[r + 1]; a++)
                    for (int bb = D.start[r]; bb < D.start[r + 1]; bb++) drow[D.col[a]][D.col[bb]] += sw * D.val[a] * D.val[bb];
            }
            for (int i = 0; i < nd; i++) drow[i][i] += (double)dt * damp_k_M * (double)mass[i];
            Ddiag.assign(nd, 0.0);
            Damp.start.assign(nd + 1, 0);
            Damp.col.clear(); Damp.val.clear();
            for (int i = 0; i < nd; i++) {
                std::vector<std::pair<int, double>> e(drow[i].begin(), drow[i].end());
                std::sort(e.begin(), e.end());
                for (auto& kv : e) {
                    arow[i][kv.first] += kv.second;
                    if (kv.first == i) Ddiag[i] = kv.second;
                    else { Damp.col.push_back(kv.first); Damp.val.push_back(kv.second); }
                }
                Damp.start[i + 1] = (int)Damp.col.size();
            }
        }
        dt2Wc.assign(nd, R(0));
        if (contact)
            for (int i = 0; i < nd; i++)
                if (is_surf[i]) dt2Wc[i] = h2 * cw[i];
        Adiag.assign(nd, R(0));
        A.start.assign(nd + 1, 0);
        A.col.clear(); A.val.clear();
        for (int i = 0; i < nd; i++) {
            std::vector<std::pair<int, double>> e(arow[i].begin(), arow[i].end());
            std::sort(e.begin(), e.end());
            double diag = (double)mass[i] + (double)dt2Wc[i];
            for (auto& kv : e) {
                if (kv.first == i) diag += kv.second;
                else { A.col.push_back(kv.first); A.val.push_back(kv.second); }
            }
            Adiag[i] = (R)diag;
            A.start[i + 1] = (int)A.col.size();
        }
        if (backend == 1) {
            std::vector<double> ad(nd);
            for (int i = 0; i < nd; i++) ad[i] = (double)Adiag[i];
            if (!chol.factor(nd, A.start, A.col, A.val, ad)) fprintf(stderr, "oracle: damped A is not positive definite\n");
        }
        DtW2.start.assign(nd + 1, 0);
        DtW2.col.clear(); DtW2.val.clear();
        for (int i = 0; i < nd; i++) {
            for (auto& kv : dtw[i]) { DtW2.col.push_back(kv.first); DtW2.val.push_back(kv.second); }
            DtW2.start[i + 1] = (int)DtW2.col.size();
        }
    }

    void reset() {
        x0 = x0_init;
        v = v0_init;
        x = x0;
        p.assign(3 * n, R(0));
        mxt.assign(3 * n, R(0));
        b.assign(3 * nd, R(0));
        Ue.assign(3 * m, R(0));
        Uc.assign(3 * nd, R(0));
        z.assign(3 * m, R(0));
        cts.clear();
        peak = 0;
    }

    // do_integration_kernel (jacobi_solver.cu:183-215)
    void pre_integration() {
        for (int i = 0; i < n; i++) {
            if (!fixed[i]) {
                if (i < nd) {
                    v[3 * i + 1] -= g * dt;
                    for (int k = 0; k < 3; k++) x[3 * i + k] = x0[3 * i + k] + v[3 * i + k] * dt;
                } else {
                    for (int k = 0; k < 3; k++) x[3 * i + k] = x0[3 * i + k];
                }
            } else {
                for (int k = 0; k < 3; k++) { v[3 * i + k] = 0; x[3 * i + k] = x0[3 * i + k]; }
            }
            for (int k = 0; k < 3; k++) mxt[3 * i + k] = mass[i] * x[3 * i + k];
        }
        // the CPU backend's b_ini = Damp x0 (admm_impl_cpu.cpp:295), part of every
        // right-hand side (:344): folded into M x~
        if (backend == 1)
            for (int i = 0; i < nd; i++)
                for (int k = 0; k < 3; k++) {
                    double a = Ddiag[i] * (double)x0[3 * i + k];
                    for (int e = Damp.start[i]; e < Damp.start[i + 1]; e++) a += Damp.val[e] * (double)x0[3 * Damp.col[e] + k];
                    mxt[3 * i + k] += (R)a;
                }
    }

    // D*x for rows [r0, r0+nr): tri/tet through F = E * Binv (edges first),
    // bending and pins through their D rows.
    void Dx_rows(std::vector<R>& out) const {
        out.assign(3 * m, R(0));
        for (int c = 0; c < ntri; c++) {
            const int* id = &tri_inds[3 * c];
            const R* B = &tri_binv[4 * c];
            R e[2][3];
            for (int k = 0; k < 3; k++) { e[0][k] = x[3 * id[1] + k] - x[3 * id[0] + k]; e[1][k] = x[3 * id[2] + k] - x[3 * id[0] + k]; }
            for (int r = 0; r < 2; r++)
                for (int k = 0; k < 3; k++) out[3 * (tri_sr + 2 * c + r) + k] = e[0][k] * B[0 * 2 + r] + e[1][k] * B[1 * 2 + r];
        }
        for (int c = 0; c < ntet; c++) {
            const int* id = &tet_inds[4 * c];
            const R* B = &tet_binv[9 * c];
            R e[3][3];
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++) e[j][k] = x[3 * id[j + 1] + k] - x[3 * id[0] + k];
            for (int r = 0; r < 3; r++)
                for (int k = 0; k < 3; k++)
                    out[3 * (tet_sr + 3 * c + r) + k] = (e[0][k] * B[0 * 3 + r] + e[1][k] * B[1 * 3 + r]) + e[2][k] * B[2 * 3 + r];
        }
        for (int c = 0; c < nbend; c++)
            for (int k = 0; k < 3; k++) {
                R s = 0;
                for (int a = bend_off[c]; a < bend_off[c + 1]; a++) s += bend_coef[a] * x[3 * bend_inds[a] + k];
                out[3 * (bend_sr + c) + k] = s;
            }
        for (int c = 0; c < npin; c++)
            for (int k = 0; k < 3; k++) out[3 * (pin_sr + c) + k] = x[3 * pin_inds[c] + k];
    }

    // z = prox(D x + Ue)  (do_project_elastic, admm_impl_gpu.cu:52-59)
    void local_step() {
        std::vector<R> dx;
        Dx_rows(dx);
        for (int i = 0; i < 3 * m; i++) z[i] = dx[i] + Ue[i];
#pragma omp parallel for schedule(static)
        for (int c = 0; c < ntet; c++) prox_tet<R>(&z[3 * (tet_sr + 3 * c)]);
#pragma omp parallel for schedule(static)
        for (int c = 0; c < ntri; c++) prox_tri<R>(&z[3 * (tri_sr + 2 * c)]);
        for (int c = 0; c < nbend; c++) prox_bend<R>(&z[3 * (bend_sr + c)], bend_rest[c]);
        for (int c = 0; c < npin; c++)
            for (int k = 0; k < 3; k++) z[3 * (pin_sr + c) + k] = pin_pos[3 * c + k];
    }

    void detect() {
        std::vector<float> xf(3 * n);
        for (int i = 0; i < 3 * n; i++) xf[i] = (float)x[i];
        std::vector<RawPair> raw;
        dcd_all(xf.data(), surf_verts, surf_tris, surf_edges, thickness, raw, semantics, nd);
        cts.resize(raw.size());
        for (size_t c = 0; c < raw.size(); c++) convert(raw[c], cts[c]);
        peak = std::max(peak, (int)cts.size());
    }

    // convert_DCD_info_kernel (contact_solver.cu:118-154)
    void convert(const RawPair& rp, Contact& ct) const {
        for (int k = 0; k < 4; k++) ct.v[k] = rp.v[k];
        const Result<float>& r = rp.r;
        for (int k = 0; k < 3; k++) ct.bary_raw[k] = r.bary[k];
        ct.type = (r.bary[2] < -1.f) ? 0 : 1;
        auto X = [&](int i) { return mk<R>(x[3 * i], x[3 * i + 1], x[3 * i + 2]); };
        V3<R> v0 = X(ct.v[0]), v1 = X(ct.v[1]), v2 = X(ct.v[2]), v3 = X(ct.v[3]);
        V3<R> c0 = mk<R>(r.closest[0].x, r.closest[0].y, r.closest[0].z);
        V3<R> c1 = mk<R>(r.closest[1].x, r.closest[1].y, r.closest[1].z);
        V3<R> pt = R(0.5) * (c0 + c1);
        ct.point[0] = pt.x; ct.point[1] = pt.y; ct.point[2] = pt.z;
        if (ct.type == 0) {
            ct.bary[0] = 1 - (R)r.bary[0]; ct.bary[1] = (R)r.bary[0]; ct.bary[2] = (R)r.bary[1] - 1; ct.bary[3] = -(R)r.bary[1];
        } else {
            ct.bary[0] = 1; ct.bary[1] = -(R)r.bary[0]; ct.bary[2] = -(R)r.bary[1]; ct.bary[3] = -(R)r.bary[2];
        }
        V3<R> nrm = ct.type == 0 ? normalized(cross(v1 - v0, v3 - v2)) : normalized(cross(v2 - v1, v3 - v1));
        V3<R> hv = c0 - c1;
        R hcn = dot(hv, nrm);
        if (hcn < 0) { nrm = R(-1) * nrm; hcn = -hcn; }
        ct.gap = hcn - (R)thickness;
        ct.normal[0] = nrm.x; ct.normal[1] = nrm.y; ct.normal[2] = nrm.z;
    }

    // compute_Scc_kernel (contact_solver.cu:188-227) with counts over all four
    // vertices (updateContactCounts, 90-101); r_c reset (240-243).
    void compute_scc(R eps, R gam) {
        int nc = (int)cts.size();
        std::vector<int> cnt(n, 0);
        for (auto& c : cts) for (int k = 0; k < 4; k++) cnt[c.v[k]]++;
        Gam.assign(4 * nc, R(0));
        Kc.assign(3 * nc, R(0));
        rc.assign(3 * nc, R(0));
        du.assign(3 * nc, R(0));
        for (int c = 0; c < nc; c++)
            scc_contact<R>(cts[c], cnt.data(), cw.data(), cwinv.data(), eps, gam, R(1) / dt, backend == 1, &Gam[4 * c],
                           &Kc[3 * c]);
        vstart.assign(n + 1, 0);
        for (int i = 0; i < n; i++) vstart[i + 1] = vstart[i] + cnt[i];
        vlist.assign(vstart[n], 0);
        std::vector<int> fill(n, 0);
        for (int c = 0; c < nc; c++)
            for (int k = 0; k < 4; k++) { int vi = cts[c].v[k]; vlist[vstart[vi] + fill[vi]++] = 4 * c + k; }
    }

    // project_impl (contact_solver.cu:402-431): warm start p += Gamma r_c, then
    // gs_max_iter x {friction-cone projection per contact, gather into p}.
    void project() {
        int nc = (int)cts.size();
        cmu.assign(nc, mu);
        if (!vmu.empty())
            for (int c = 0; c < nc; c++) {
                int k = 0;
                while (k < 3 && cts[c].v[k] >= nd) k++;
                cmu[c] = vmu[cts[c].v[k]];
            }
        for (int c = 0; c < nc; c++)
            for (int k = 0; k < 4; k++) {
                int vi = cts[c].v[k];
                if (vi < nd) for (int a = 0; a < 3; a++) p[3 * vi + a] += Gam[4 * c + k] * rc[3 * c + a];
            }
        if (backend == 1) {
            project_gs_serial(nc);
            return;
        }
        for (int it = 0; it < gs_max_iter; it++) {
            for (int c = 0; c < nc; c++) cone_step<R>(cts[c], cmu[c], p.data(), &Kc[3 * c], &rc[3 * c], &du[3 * c]);
            gather_p<R>(nd, vstart.data(), vlist.data(), Gam.data(), du.data(), p.data());
        }
    }

    // b = M x~ + h^2 D^T W^2 (z - Ue) + h^2 W_c (h p + x0 - Uc)  (admm_impl_gpu.cu:307-318)
    void rhs() {
        for (int i = 0; i < nd; i++)
            for (int k = 0; k < 3; k++) {
                R s = 0;
                for (int a = DtW2.start[i]; a < DtW2.start[i + 1]; a++) {
                    int r = DtW2.col[a];
                    s += (R)DtW2.val[a] * (z[3 * r + k] - Ue[3 * r + k]);
                }
                R bi = mxt[3 * i + k] + s;
                if (contact) bi = bi + dt2Wc[i] * ((p[3 * i + k] * dt + x0[3 * i + k]) - Uc[3 * i + k]);
                b[3 * i + k] = bi;
            }
    }

    // cu_jacobi_global (jacobi_solver.cu:141-180)
    void jacobi(int sweeps) {
        std::vector<R> xn(3 * nd);
        for (int s = 0; s < sweeps; s++) {
            jacobi_sweep<R>(nd, A.start.data(), A.col.data(), A.val.data(), Adiag.data(), b.data(), x.data(), xn.data());
            for (int i = 0; i < 3 * nd; i++) x[i] = xn[i];
        }
    }

    // The CPU backend's projection after the warm start: gs_max_iter serial
    // Gauss-Seidel sweeps in contact-list order, each contact's update scattered into
    // p at once (_project_feasible_plain / _project_one_contact, admm_impl_cpu.cpp:390-448).
    void project_gs_serial(int nc) {
        for (int it = 0; it < gs_max_iter; it++)
            for (int c = 0; c < nc; c++) {
                const Contact& ct = cts[c];
                R u[3];
                for (int a = 0; a < 3; a++)
                    u[a] = (((R)ct.bary[0] * p[3 * ct.v[0] + a] + (R)ct.bary[1] * p[3 * ct.v[1] + a]) +
                            (R)ct.bary[2] * p[3 * ct.v[2] + a]) + (R)ct.bary[3] * p[3 * ct.v[3] + a] + Kc[3 * c + a];
                R nrm[3] = {(R)ct.normal[0], (R)ct.normal[1], (R)ct.normal[2]};
                R us[3];
                for (int a = 0; a < 3; a++) us[a] = u[a] - rc[3 * c + a];
                R uN = (nrm[0] * us[0] + nrm[1] * us[1]) + nrm[2] * us[2];
                R uT[3];
                for (int a = 0; a < 3; a++) uT[a] = us[a] - uN * nrm[a];
                if (uN < 0) {
                    R tau = std::sqrt((uT[0] * uT[0] + uT[1] * uT[1]) + uT[2] * uT[2]);
                    R alpha = -cmu[c] * uN;
                    uN = 0;
                    if (tau <= alpha) uT[0] = uT[1] = uT[2] = 0;
                    else { R s = R(1) - alpha / tau; for (int a = 0; a < 3; a++) uT[a] = s * uT[a]; }
                }
                R d[3];
                for (int a = 0; a < 3; a++) {
                    d[a] = (uN * nrm[a] + uT[a]) - u[a];
                    rc[3 * c + a] = rc[3 * c + a] + d[a];
                }
                for (int k = 0; k < 4; k++) {
                    const int vi = ct.v[k];
                    if (vi < nd) for (int a = 0; a < 3; a++) p[3 * vi + a] += Gam[4 * c + k] * d[a];
                }
            }
    }

    // The CPU backend's exact global solve of the damped A, column by column.
    void exact_solve() {
        std::vector<double> bc(nd), xc(nd);
        for (int k = 0; k < 3; k++) {
            for (int i = 0; i < nd; i++) bc[i] = (double)b[3 * i + k];
            chol.solve(bc.data(), xc.data());
            for (int i = 0; i < nd; i++) x[3 * i + k] = (R)xc[i];
        }
    }

    // Global step with preconditioned CG (global_solver > 0; no reference
    // counterpart): Chronopoulos-Gear PCG on A (x) I3 over the 3 nd unknowns,
    // warm-started from x, `iters` updates, the same recurrences as the GPU
    // kernels (k_pcg_init / k_pcg_spmv / k_pcg_update), dot products in FP64.
    void apply_A(const std::vector<R>& v, std::vector<R>& out) {
        for (int i = 0; i < nd; i++)
            for (int k = 0; k < 3; k++) {
                R acc = 0;
                for (int a = A.start[i]; a < A.start[i + 1]; a++) acc += v[3 * A.col[a] + k] * (R)A.val[a];
                out[3 * i + k] = acc + Adiag[i] * v[3 * i + k];
            }
    }
    void precond(const std::vector<R>& r, std::vector<R>& u) {
        for (int i = 0; i < nd; i++) {
            if (global_solver == 2 && !pblock.empty()) {
                const R* B = &pblock[9 * i];
                for (int k = 0; k < 3; k++)
                    u[3 * i + k] = B[3 * k] * r[3 * i] + B[3 * k + 1] * r[3 * i + 1] + B[3 * k + 2] * r[3 * i + 2];
            } else {
                for (int k = 0; k < 3; k++) u[3 * i + k] = r[3 * i + k] / Adiag[i];
            }
        }
    }
    void pcg(int iters) {
        const int N = 3 * nd;
        std::vector<R> r(N), u(N), w(N), pv(N, R(0)), sv(N, R(0)), ax(N);
        apply_A(x, ax);
        for (int i = 0; i < N; i++) r[i] = b[i] - ax[i];
        precond(r, u);
        double gamma_prev = 0, alpha_prev = 0;
        for (int it = 0; it < iters; it++) {
            apply_A(u, w);
            double gamma = 0, delta = 0;
            for (int i = 0; i < N; i++) {
                gamma += (double)r[i] * (double)u[i];
                delta += (double)w[i] * (double)u[i];
            }
            double alpha, beta;
            if (it == 0) {
                beta = 0;
                alpha = delta != 0 ? gamma / delta : 0;
            } else {
                beta = gamma_prev != 0 ? gamma / gamma_prev : 0;
                const double den = delta - beta * gamma / (alpha_prev != 0 ? alpha_prev : 1.0);
                alpha = den != 0 ? gamma / den : 0;
            }
            gamma_prev = gamma;
            alpha_prev = alpha;
            const R a = (R)alpha, bt = (R)beta;
            for (int i = 0; i < N; i++) {
                pv[i] = u[i] + bt * pv[i];
                sv[i] = w[i] + bt * sv[i];
                x[i] = x[i] + a * pv[i];
                r[i] = r[i] - a * sv[i];
            }
            precond(r, u);
        }
    }

    void global_solve() {
        if (backend == 1) exact_solve();
        else if (global_solver > 0) pcg(pcg_iter);
        else jacobi(jacobi_iter);
    }

    // Learned global step (the GPU's k_rhs_learn / k_lsweep / k_ljudge / k_ldecide):
    // warm start x += theta (x - xl) unless first, xl <- x received; K sweeps
    // x_{k+1} = x_k + omega_k m (b - A x_k) + beta_k (x_k - x_{k-1}); the solve fails
    // when |b - A x_K|^2 > |b - A x_c|^2 (x_c the received iterate) and |b - A x_K| >
    // 1e-5 |b| (FP64 sums), and a failed solve is replaced by the plain one: x <- x_c,
    // jacobi_iter sweeps.  The warm start restarts adaptively: once a warm start raised
    // the residual (|b - A x_0| > |b - A x_c|) it stays off until the next substep.
    void learned_solve(bool first) {
        const int N = 3 * nd;
        if (learn_K == 0) {  // defaults: the Jacobi sweep
            learn_K = std::max(1, jacobi_iter);
            learn_omega.assign(learn_K, R(1));
            learn_beta.assign(learn_K, R(0));
            learn_m.resize(nd);
            for (int i = 0; i < nd; i++) learn_m[i] = R(1) / Adiag[i];
            learn_theta.assign(nd, R(0));
        }
        if ((int)xl.size() != N) xl.assign(N, R(0));
        if (first) warm_on = true;
        const bool extrap = !first && warm_on;
        for (int i = 0; i < nd; i++)
            for (int k = 0; k < 3; k++) {
                const R xi = x[3 * i + k], xo = xl[3 * i + k];
                xl[3 * i + k] = xi;
                if (extrap) x[3 * i + k] = learn_theta[i] * (xi - xo) + xi;
            }
        std::vector<R> xp(x.begin(), x.begin() + N), xn(N), ax(N);
        double r0 = 0, rx0 = 0, rK = 0, bb = 0;
        for (int q = 0; q < N; q++) bb += (double)b[q] * (double)b[q];
        if (extrap) {  // the received iterate's residual (x_0 = x_c without a warm start)
            std::vector<R> xc(x.begin(), x.end()), axc(N);
            std::copy(xl.begin(), xl.end(), xc.begin());
            apply_A(xc, axc);
            for (int q = 0; q < N; q++) {
                const R r = b[q] - axc[q];
                r0 += (double)r * (double)r;
            }
        }
        for (int s = 0; s < learn_K; s++) {
            apply_A(x, ax);
            for (int i = 0; i < nd; i++)
                for (int k = 0; k < 3; k++) {
                    const int q = 3 * i + k;
                    const R r = b[q] - ax[q];
                    if (s == 0) rx0 += (double)r * (double)r;
                    const R bt = s == 0 ? R(0) : learn_beta[s];
                    xn[q] = (learn_omega[s] * learn_m[i]) * r + (bt * (x[q] - xp[q]) + x[q]);
                }
            for (int q = 0; q < N; q++) {
                xp[q] = x[q];
                x[q] = xn[q];
            }
        }
        apply_A(x, ax);
        for (int q = 0; q < N; q++) {
            const R r = b[q] - ax[q];
            rK += (double)r * (double)r;
        }
        if (!extrap) r0 = rx0;
        // adaptive restart: a warm start that raised the residual stays off for the substep
        if (extrap && rx0 > r0) warm_on = false;
        learn_solves++;
        if (!(rK <= r0 || rK <= 1e-10 * bb)) {
            learn_failed++;
            learn_fallbacks++;
            std::copy(xl.begin(), xl.end(), x.begin());
            jacobi(jacobi_iter);
        }
    }

    // Residuals after the global solve of an iteration, before its dual update:
    //   primal^2 = sum w^2 |D x - z|^2 + sum w_c |x - x0 - h p|^2
    //   dual^2   = sum w^2 |D (x - x_prev)|^2 + sum w_c |x - x_prev|^2
    //   scale^2  = sum w^2 |z|^2 + sum w_c |x - x0|^2
    // (x_prev = x before the solve; contact terms on the dynamic contact surface).
    void residual_accumulate(double& prim, double& dual, double& den, const std::vector<R>& dx,
                             const std::vector<R>& dxprev) {
        prim = dual = den = 0;
        for (int r = 0; r < m; r++) {
            double w2 = (double)wrow[r] * (double)wrow[r];
            for (int k = 0; k < 3; k++) {
                double rp = (double)dx[3 * r + k] - (double)z[3 * r + k];
                double rd = (double)dx[3 * r + k] - (double)dxprev[3 * r + k];
                prim += w2 * rp * rp;
                dual += w2 * rd * rd;
                den += w2 * (double)z[3 * r + k] * (double)z[3 * r + k];
            }
        }
        if (contact)
            for (int i = 0; i < nd; i++) {
                if (!is_surf[i]) continue;
                double w = (double)cw[i];
                for (int k = 0; k < 3; k++) {
                    double d0 = (double)x[3 * i + k] - (double)x0[3 * i + k];
                    double rp = d0 - (double)dt * (double)p[3 * i + k];
                    double rd = (double)x[3 * i + k] - (double)xprev[3 * i + k];
                    prim += w * rp * rp;
                    dual += w * rd * rd;
                    den += w * d0 * d0;
                }
            }
    }

    // A substep (with the learned global step: every solve judged, a failed one replaced).
    int step() {
        if (global_solver != 3) return step_once(false);
        learn_substeps++;
        return step_once(true);
    }

    // ADMMImplGPU::step (admm_impl_gpu.cu:256-344)
    int step_once(bool learned) {
        const R eps = R(1) / (dt * dt * kappa + dt * beta);
        const R gam = dt * kappa / (dt * kappa + beta);
        pre_integration();
        if (!ws_ue) std::fill(Ue.begin(), Ue.end(), R(0));
        if (!ws_uc) std::fill(Uc.begin(), Uc.end(), R(0));
        // p <- v on the static range (admm_impl_gpu.cu:282)
        for (int i = 3 * nd; i < 3 * n; i++) p[i] = v[i];
        const R dt_inv = R(1) / dt;
        bool need_scc = false;
        int iters = 0;
        for (int it = 0; it < admm_max_iter; it++) {
            if (contact && it % dcd_interval == 0) { detect(); need_scc = true; }
            local_step();
            if (contact) {
                for (int i = 0; i < nd; i++)
                    for (int k = 0; k < 3; k++) p[3 * i + k] = ((x[3 * i + k] - x0[3 * i + k]) + Uc[3 * i + k]) * dt_inv;
                if (need_scc) { compute_scc(eps, gam); need_scc = false; }
                project();
            }
            rhs();
            xprev = x;
            std::vector<R> dxprev;
            Dx_rows(dxprev);
            if (learned) learned_solve(it == 0);
            else global_solve();
            std::vector<R> dx;
            Dx_rows(dx);
            double prim, dual, den;
            residual_accumulate(prim, dual, den, dx, dxprev);
            den = std::sqrt(den) + 1e-30;
            last_primal = std::sqrt(prim) / den;
            last_dual = std::sqrt(dual) / den;
            for (int i = 0; i < 3 * m; i++) Ue[i] = (dx[i] - z[i]) + Ue[i];
            if (contact)
                for (int i = 0; i < nd; i++)
                    for (int k = 0; k < 3; k++)
                        Uc[3 * i + k] = Uc[3 * i + k] + ((x[3 * i + k] - x0[3 * i + k]) - p[3 * i + k] * dt);
            iters++;
            // residual_tol > 0: test after every chunk of iterations; stop when both
            // relative residuals are within tol or another chunk would pass max_iter
            if (residual_tol > 0.f && iters % chunk == 0) {
                const bool conv = last_primal <= (double)residual_tol && last_dual <= (double)residual_tol;
                if (conv || iters + chunk > admm_max_iter) break;
            }
        }
        // do_post_process_kernel (jacobi_solver.cu:236-252)
        for (int i = 0; i < n; i++)
            for (int k = 0; k < 3; k++) {
                if (i < nd) v[3 * i + k] = (x[3 * i + k] - x0[3 * i + k]) * dt_inv;
                x0[3 * i + k] = x[3 * i + k];
            }
        return iters;
    }
};

struct Handle {
    int prec;
    Oracle<double>* d = nullptr;
    Oracle<float>* f = nullptr;
};

template <class R> static std::vector<R>* buf_of(Oracle<R>* o, int which) {
    switch (which) {
        case ADMM_BUF_X: return &o->x;
        case ADMM_BUF_X0: return &o->x0;
        case ADMM_BUF_V: return &o->v;
        case ADMM_BUF_P: return &o->p;
        case ADMM_BUF_UC: return &o->Uc;
        case ADMM_BUF_UE: return &o->Ue;
        case ADMM_BUF_Z: return &o->z;
        case ADMM_BUF_B: return &o->b;
        case ADMM_BUF_MXT: return &o->mxt;
    }
    return nullptr;
}

}  // namespace

template <class R>
static void set_learned_impl(Oracle<R>* o, int K, const float* om, const float* be, const float* m, const float* th) {
    o->learn_K = K;
    o->learn_omega.assign(om, om + K);
    o->learn_beta.assign(be, be + K);
    o->learn_beta[0] = R(0);
    o->learn_m.resize(o->nd);
    o->learn_theta.assign(o->nd, R(0));
    for (int i = 0; i < o->nd; i++) {
        o->learn_m[i] = m ? (R)m[i] : R(1) / o->Adiag[i];
        if (th) o->learn_theta[i] = (R)th[i];
    }
}
extern "C" {

void* orc_create(const AdmmB200Desc* d, int use_double) {
    Handle* h = new Handle;
    h->prec = use_double ? 64 : 32;
    if (use_double) { h->d = new Oracle<double>; h->d->setup(d); }
    else { h->f = new Oracle<float>; h->f->setup(d); }
    return h;
}

void orc_destroy(void* hp) {
    Handle* h = (Handle*)hp;
    delete h->d;
    delete h->f;
    delete h;
}

int orc_step(void* hp, int nsteps, double* primal, double* dual, int* ncontacts) {
    Handle* h = (Handle*)hp;
    int it = 0;
    for (int s = 0; s < nsteps; s++) it = h->d ? h->d->step() : h->f->step();
    if (primal) *primal = h->d ? h->d->last_primal : h->f->last_primal;
    if (dual) *dual = h->d ? h->d->last_dual : h->f->last_dual;
    if (ncontacts) *ncontacts = h->d ? (int)h->d->cts.size() : (int)h->f->cts.size();
    return it;
}

void orc_reset(void* hp) {
    Handle* h = (Handle*)hp;
    if (h->d) h->d->reset(); else h->f->reset();
}

// Copy a state buffer out (rows of 3 doubles) / in.
int orc_read(void* hp, int which, double* out, int nrows) {
    Handle* h = (Handle*)hp;
    if (h->d) {
        auto* b = buf_of(h->d, which);
        if (!b || (int)b->size() < 3 * nrows) return -1;
        for (int i = 0; i < 3 * nrows; i++) out[i] = (*b)[i];
    } else {
        auto* b = buf_of(h->f, which);
        if (!b || (int)b->size() < 3 * nrows) return -1;
        for (int i = 0; i < 3 * nrows; i++) out[i] = (*b)[i];
    }
    return 0;
}

int orc_write(void* hp, int which, const double* in, int nrows) {
    Handle* h = (Handle*)hp;
    if (h->d) {
        auto* b = buf_of(h->d, which);
        if (!b || (int)b->size() < 3 * nrows) return -1;
        for (int i = 0; i < 3 * nrows; i++) (*b)[i] = in[i];
    } else {
        auto* b = buf_of(h->f, which);
        if (!b || (int)b->size() < 3 * nrows) return -1;
        for (int i = 0; i < 3 * nrows; i++) (*b)[i] = (float)in[i];
    }
    return 0;
}

void orc_local_step(void* hp) {
    Handle* h = (Handle*)hp;
    if (h->d) h->d->local_step(); else h->f->local_step();
}
void orc_pre_integration(void* hp) {
    Handle* h = (Handle*)hp;
    if (h->d) h->d->pre_integration(); else h->f->pre_integration();
}
void orc_rhs(void* hp) {
    Handle* h = (Handle*)hp;
    if (h->d) h->d->rhs(); else h->f->rhs();
}
void orc_jacobi(void* hp, int sweeps) {
    Handle* h = (Handle*)hp;
    if (h->d) h->d->jacobi(sweeps); else h->f->jacobi(sweeps);
}

// The constant global-step matrix: nnz of the off-diagonal CSR (when start is
// null), else start[nd+1], col[nnz], val[nnz] and diag[nd] (FP64 oracle).
int orc_system(void* hp, int32_t* start, int32_t* col, double* val, double* diag) {
    Handle* h = (Handle*)hp;
    if (!h->d) return -1;
    const auto& o = *h->d;
    if (!start) return (int)o.A.col.size();
    for (size_t i = 0; i < o.A.start.size(); i++) start[i] = o.A.start[i];
    for (size_t k = 0; k < o.A.col.size(); k++) {
        col[k] = o.A.col[k];
        val[k] = o.A.val[k];
    }
    for (int i = 0; i < o.nd; i++) diag[i] = o.Adiag[i];
    return (int)o.A.col.size();
}

void orc_pcg(void* hp, int iters) {
    Handle* h = (Handle*)hp;
    if (h->d) h->d->pcg(iters); else h->f->pcg(iters);
}

// Learned global step (global_solver 3): K coefficient pairs, per-vertex m and theta
// (null: 1 / a_ii and 0).
void orc_set_learned(void* hp, int K, const float* om, const float* be, const float* m, const float* th) {
    auto* h = static_cast<Handle*>(hp);
    if (h->d) set_learned_impl(h->d, K, om, be, m, th);
    else set_learned_impl(h->f, K, om, be, m, th);
}
// Rest-shape records computed by the oracle itself from the mesh (FP64 from the float
// positions), independent of the scene builder that feeds both the oracle and the GPU:
// triangles (TriangleConstraint ctor, triangle_constraint.h:41-58): orthonormal basis
// n1 = e12/|e12|, n2 = normalised e13 - (e13.n1) n1, Binv = (basis^T [e12 e13])^-1
// (row-major 2x2), area = det / 2;  tets (tetrahedral_constraint.h:41-51): Binv =
// [e12 e13 e14]^-1 (row-major 3x3), volume = |det| / 6;  lumped mass
// (MeshData::get_mass, mesh_container.h:452-472): area/3 and volume/4 times the density.
void orc_tri_rest(const float* v, const int32_t* tri, int ntri, double* binv4, double* area) {
    for (int c = 0; c < ntri; c++) {
        const int* id = &tri[3 * c];
        double e12[3], e13[3];
        for (int k = 0; k < 3; k++) {
            e12[k] = (double)v[3 * id[1] + k] - (double)v[3 * id[0] + k];
            e13[k] = (double)v[3 * id[2] + k] - (double)v[3 * id[0] + k];
        }
        const double l1 = std::sqrt(e12[0] * e12[0] + e12[1] * e12[1] + e12[2] * e12[2]);
        double n1[3] = {e12[0] / l1, e12[1] / l1, e12[2] / l1};
        const double d = e13[0] * n1[0] + e13[1] * n1[1] + e13[2] * n1[2];
        double n2[3] = {e13[0] - d * n1[0], e13[1] - d * n1[1], e13[2] - d * n1[2]};
        const double l2 = std::sqrt(n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]);
        for (int k = 0; k < 3; k++) n2[k] /= l2;
        auto dot3 = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
        const double M[2][2] = {{dot3(n1, e12), dot3(n1, e13)}, {dot3(n2, e12), dot3(n2, e13)}};
        const double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        binv4[4 * c + 0] = M[1][1] / det;
        binv4[4 * c + 1] = -M[0][1] / det;
        binv4[4 * c + 2] = -M[1][0] / det;
        binv4[4 * c + 3] = M[0][0] / det;
        area[c] = det / 2.0;
    }
}

void orc_tet_rest(const float* v, const int32_t* tet, int ntet, double* binv9, double* vol) {
    for (int c = 0; c < ntet; c++) {
        const int* id = &tet[4 * c];
        double B[3][3];  // columns e12, e13, e14
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) B[k][j] = (double)v[3 * id[j + 1] + k] - (double)v[3 * id[0] + k];
        const double c00 = B[1][1] * B[2][2] - B[1][2] * B[2][1], c01 = B[1][2] * B[2][0] - B[1][0] * B[2][2],
                     c02 = B[1][0] * B[2][1] - B[1][1] * B[2][0];
        const double det = B[0][0] * c00 + B[0][1] * c01 + B[0][2] * c02;
        const double inv[3][3] = {
            {c00 / det, (B[0][2] * B[2][1] - B[0][1] * B[2][2]) / det, (B[0][1] * B[1][2] - B[0][2] * B[1][1]) / det},
            {c01 / det, (B[0][0] * B[2][2] - B[0][2] * B[2][0]) / det, (B[0][2] * B[1][0] - B[0][0] * B[1][2]) / det},
            {c02 / det, (B[0][1] * B[2][0] - B[0][0] * B[2][1]) / det, (B[0][0] * B[1][1] - B[0][1] * B[1][0]) / det}};
        for (int r = 0; r < 3; r++)
            for (int k = 0; k < 3; k++) binv9[9 * c + 3 * r + k] = inv[r][k];
        vol[c] = std::fabs(det / 6.0);
    }
}

void orc_lumped_mass(int n, const float* v, const int32_t* tri, int ntri, const double* tri_density,
                     const int32_t* tet, int ntet, const double* tet_density, double* mass) {
    std::vector<double> a(ntri), b4(4 * (size_t)ntri), vo(ntet), b9(9 * (size_t)ntet);
    if (ntri) orc_tri_rest(v, tri, ntri, b4.data(), a.data());
    if (ntet) orc_tet_rest(v, tet, ntet, b9.data(), vo.data());
    for (int i = 0; i < n; i++) mass[i] = 0.0;
    for (int f = 0; f < ntri; f++)
        for (int k = 0; k < 3; k++) mass[tri[3 * f + k]] += a[f] / 3.0 * tri_density[f];
    for (int t = 0; t < ntet; t++)
        for (int k = 0; k < 4; k++) mass[tet[4 * t + k]] += vo[t] / 4.0 * tet_density[t];
}

void orc_learned_stats(void* hp, long long* out4) {
    auto* h = static_cast<Handle*>(hp);
    if (h->d) {
        out4[0] = h->d->learn_substeps; out4[1] = h->d->learn_fallbacks;
        out4[2] = h->d->learn_solves; out4[3] = h->d->learn_failed;
    } else {
        out4[0] = h->f->learn_substeps; out4[1] = h->f->learn_fallbacks;
        out4[2] = h->f->learn_solves; out4[3] = h->f->learn_failed;
    }
}

// Learned preconditioner blocks (9 per dynamic vertex, row-major) for global_solver 2.
void orc_set_preconditioner(void* hp, const float* blocks, int nd) {
    Handle* h = (Handle*)hp;
    if (h->d) h->d->pblock.assign(blocks, blocks + 9 * (size_t)nd);
    else h->f->pblock.assign(blocks, blocks + 9 * (size_t)nd);
}

// The contact sub-problem on the last detection, from the current x, x0, Uc:
// compute_Scc, p = (x - x0 + Uc)/h, warm start and gs_max_iter projections.
void orc_contact_step(void* hp) {
    Handle* h = (Handle*)hp;
    auto run = [](auto* o) {
        using R = std::remove_reference_t<decltype(o->dt)>;
        const R eps = R(1) / (o->dt * o->dt * o->kappa + o->dt * o->beta);
        const R gam = o->dt * o->kappa / (o->dt * o->kappa + o->beta);
        const R dt_inv = R(1) / o->dt;
        for (int i = 0; i < o->nd; i++)
            for (int k = 0; k < 3; k++)
                o->p[3 * i + k] = ((o->x[3 * i + k] - o->x0[3 * i + k]) + o->Uc[3 * i + k]) * dt_inv;
        o->compute_scc(eps, gam);
        o->project();
    };
    if (h->d) run(h->d); else run(h->f);
}

// Run DCD + contact conversion on the handle's current x.
int orc_detect(void* hp) {
    Handle* h = (Handle*)hp;
    if (h->d) { h->d->detect(); return (int)h->d->cts.size(); }
    h->f->detect();
    return (int)h->f->cts.size();
}

// Contacts of the last detection: pairs (int4), bary (4), normal (3), point (3), gap.
int orc_contacts(void* hp, int32_t* pairs, double* bary, double* normal, double* point, double* gap, int cap) {
    Handle* h = (Handle*)hp;
    const std::vector<Contact>& c = h->d ? h->d->cts : h->f->cts;
    int nc = std::min((int)c.size(), cap);
    for (int i = 0; i < nc; i++) {
        for (int k = 0; k < 4; k++) pairs[4 * i + k] = c[i].v[k];
        if (bary) for (int k = 0; k < 4; k++) bary[4 * i + k] = c[i].bary[k];
        if (normal) for (int k = 0; k < 3; k++) normal[3 * i + k] = c[i].normal[k];
        if (point) for (int k = 0; k < 3; k++) point[3 * i + k] = c[i].point[k];
        if (gap) gap[i] = c[i].gap;
    }
    return (int)c.size();
}

// Standalone DCD on float positions (for pair-set parity): returns the pair count;
// fills up to cap int4 pairs.
int orc_dcd2(const float* x, int n, const int32_t* sv, int nsv, const int32_t* st, int nst,
             const int32_t* se, int nse, float thickness, int32_t* pairs, float* dist, int cap,
             int semantics, int static_begin) {
    (void)n;
    std::vector<int> SV(sv, sv + nsv), ST(st, st + 3 * nst), SE(se, se + 2 * nse);
    std::vector<RawPair> raw;
    dcd_all(x, SV, ST, SE, thickness, raw, semantics, static_begin);
    int nc = std::min((int)raw.size(), cap);
    for (int i = 0; i < nc; i++) {
        for (int k = 0; k < 4; k++) pairs[4 * i + k] = raw[i].v[k];
        if (dist) dist[i] = raw[i].r.distance;
    }
    return (int)raw.size();
}

int orc_dcd(const float* x, int n, const int32_t* sv, int nsv, const int32_t* st, int nst,
            const int32_t* se, int nse, float thickness, int32_t* pairs, float* dist, int cap) {
    return orc_dcd2(x, n, sv, nsv, st, nst, se, nse, thickness, pairs, dist, cap, 0, 1 << 30);
}

// Unit-level functions (float and double) for known-answer tests.
void orc_svd3_d(const double* F, double* U, double* S, double* V) {
    M3<double> f, u, v;
    for (int i = 0; i < 9; i++) f.a[i / 3][i % 3] = F[i];
    svd3(f, u, S, v);
    for (int i = 0; i < 9; i++) { U[i] = u.a[i / 3][i % 3]; V[i] = v.a[i / 3][i % 3]; }
}
void orc_prox_tet_d(double* z) { prox_tet<double>(z); }
void orc_prox_tri_d(double* z) { prox_tri<double>(z); }
void orc_prox_tet_f(float* z) { prox_tet<float>(z); }
void orc_prox_tri_f(float* z) { prox_tri<float>(z); }
// out: distance, sqrDistance, bary[3], closest0[3], closest1[3]  (11 floats)
void orc_dcd_pt_f(const float* p, const float* t0, const float* t1, const float* t2, float* out) {
    Result<float> r = dcd_pt(mk(p[0], p[1], p[2]), mk(t0[0], t0[1], t0[2]), mk(t1[0], t1[1], t1[2]), mk(t2[0], t2[1], t2[2]));
    float o[11] = {r.distance, r.sqrDistance, r.bary[0], r.bary[1], r.bary[2],
                   r.closest[0].x, r.closest[0].y, r.closest[0].z, r.closest[1].x, r.closest[1].y, r.closest[1].z};
    std::memcpy(out, o, sizeof(o));
}
static void pack11(const Result<float>& r, float* out) {
    float o[11] = {r.distance, r.sqrDistance, r.bary[0], r.bary[1], r.bary[2],
                   r.closest[0].x, r.closest[0].y, r.closest[0].z, r.closest[1].x, r.closest[1].y, r.closest[1].z};
    std::memcpy(out, o, sizeof(o));
}
void orc_gt_pt_f(const float* p, const float* t0, const float* t1, const float* t2, float* out) {
    pack11(gt_point_triangle(mk(p[0], p[1], p[2]), mk(t0[0], t0[1], t0[2]), mk(t1[0], t1[1], t1[2]),
                             mk(t2[0], t2[1], t2[2])), out);
}
void orc_gt_ee_f(const float* p0, const float* p1, const float* q0, const float* q1, float* out) {
    pack11(gt_segment_segment(mk(p0[0], p0[1], p0[2]), mk(p1[0], p1[1], p1[2]), mk(q0[0], q0[1], q0[2]),
                              mk(q1[0], q1[1], q1[2])), out);
}
void orc_dcd_ee_f(const float* p0, const float* p1, const float* q0, const float* q1, float* out) {
    Result<float> r = dcd_ee(mk(p0[0], p0[1], p0[2]), mk(p1[0], p1[1], p1[2]), mk(q0[0], q0[1], q0[2]), mk(q1[0], q1[1], q1[2]));
    float o[11] = {r.distance, r.sqrDistance, r.bary[0], r.bary[1], r.bary[2],
                   r.closest[0].x, r.closest[0].y, r.closest[0].z, r.closest[1].x, r.closest[1].y, r.closest[1].z};
    std::memcpy(out, o, sizeof(o));
}

int orc_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// The shared pieces on caller-given arrays (FP32), for pinning against the reference's
// kernels.  Contacts: v4 [nc x 4], bary4 [nc x 4], normal3 [nc x 3], gap [nc].
static Contact make_contact(const int* v4, const float* bary4, const float* normal3, float gap) {
    Contact ct{};
    for (int k = 0; k < 4; k++) {
        ct.v[k] = v4[k];
        ct.bary[k] = bary4[k];
    }
    for (int k = 0; k < 3; k++) ct.normal[k] = normal3[k];
    ct.gap = gap;
    return ct;
}

void orc_scc_f(int nc, const int* v4, const float* bary4, const float* gap, const float* normal3, const int* cnt,
               const float* w, const float* winv, float eps, float gam, float dt_inv, float* Gam4, float* Kc3) {
    for (int c = 0; c < nc; c++)
        scc_contact<float>(make_contact(v4 + 4 * c, bary4 + 4 * c, normal3 + 3 * c, gap[c]), cnt, w, winv, eps, gam,
                           dt_inv, false, Gam4 + 4 * c, Kc3 + 3 * c);
}

void orc_cone_step_f(int nc, const float* mu, const int* v4, const float* bary4, const float* normal3, const float* p,
                     const float* Kc3, float* rc3, float* du3) {
    for (int c = 0; c < nc; c++)
        cone_step<float>(make_contact(v4 + 4 * c, bary4 + 4 * c, normal3 + 3 * c, 0.f), mu[c], p, Kc3 + 3 * c,
                         rc3 + 3 * c, du3 + 3 * c);
}

void orc_gather_p_f(int nv, const int* vstart, const int* vlist, const float* Gam4, const float* du3, float* p) {
    gather_p<float>(nv, vstart, vlist, Gam4, du3, p);
}

void orc_jacobi_sweep_f(int rows, const int* start, const int* col, const float* val, const float* diag, const float* b,
                        const float* x, float* xn) {
    jacobi_sweep<float, float>(rows, start, col, val, diag, b, x, xn);
}

}  // extern "C"
