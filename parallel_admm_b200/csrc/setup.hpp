// setup.hpp -- host-side assembly for one scene (ADMMImplGPU::precompute,
// admm_impl_gpu.cu:157-254): the D rows of every constraint, the constant
// system matrix A = M + h^2 D^T W^2 D + h^2 W_c split into diagonal and a
// sliced-ELL off-diagonal part, and h^2 D^T W^2 as a sliced-ELL gather.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "admm_b200.h"

namespace admm {

struct HostEll {
    int rows = 0, nslices = 0, lanes = 1;
    std::vector<int> ptr, col;
    std::vector<float> val;
    std::vector<int> rowid;  // [nslices * S] row of each slot (empty: slot = row)
    int64_t nnz = 0;  // true entries (without padding)
};

struct HostCsr {
    std::vector<int> start, col;
    std::vector<double> val;
};

// Sliced ELL with T lanes per row (T in {1, 2, 4, 8}): slices of S = 32/T rows,
// each slice's width padded to a multiple of T.  Entry k of local row lr of
// slice s sits at ptr[s] + (k / T) * 32 + (k % T) * S + lr, so one warp step
// reads 32 consecutive entries.  Padding repeats the row's own column with a
// zero value (branch-free in the kernel).  T = 1 is the classic sliced ELL of
// Monakov et al. (2010) with slice height 32.
// permute: within each window of 32 consecutive rows the rows are placed in the
// slots in order of decreasing length (ties by index), so that rows of similar
// length share a slice and the padding shrinks (the vertices of a tet lattice
// alternate between 6 and 18 neighbours, which pads every unpermuted slice to
// 18); rowid[slot] gives the row, rows for the empty slots past the end.  A
// window never straddles a multiple of 32, so row ranges that start at such
// multiples own exactly their slices.  Each row keeps its entries, their order
// and lane layout, so its sum is the same as without the permutation.
inline HostEll csr_to_sliced_ell(const HostCsr& c, int rows, int T, bool permute = false) {
    HostEll e;
    const int S = 32 / T;
    e.rows = rows;
    e.lanes = T;
    e.nslices = (rows + S - 1) / S;
    std::vector<int> order((size_t)e.nslices * S, rows);
    for (int r = 0; r < rows; r++) order[r] = r;
    if (permute) {
        auto len = [&](int r) { return c.start[r + 1] - c.start[r]; };
        for (int w0 = 0; w0 < rows; w0 += 32) {
            const int w1 = std::min(rows, w0 + 32);
            std::stable_sort(order.begin() + w0, order.begin() + w1, [&](int a, int b) { return len(a) > len(b); });
        }
        e.rowid = order;
    }
    e.ptr.assign(e.nslices + 1, 0);
    for (int s = 0; s < e.nslices; s++) {
        int w = 0;
        for (int k = s * S; k < (s + 1) * S; k++)
            if (order[k] < rows) w = std::max(w, c.start[order[k] + 1] - c.start[order[k]]);
        w = (w + T - 1) / T * T;
        e.ptr[s + 1] = e.ptr[s] + w * S;
    }
    e.col.assign(e.ptr[e.nslices], 0);
    e.val.assign(e.ptr[e.nslices], 0.f);
    for (int s = 0; s < e.nslices; s++) {
        const int w = (e.ptr[s + 1] - e.ptr[s]) / S;
        for (int lr = 0; lr < S; lr++) {
            const int r = order[s * S + lr];
            const int len = r < rows ? c.start[r + 1] - c.start[r] : 0;
            for (int k = 0; k < w; k++) {
                const int idx = e.ptr[s] + (k / T) * 32 + (k % T) * S + lr;
                if (k < len) {
                    e.col[idx] = c.col[c.start[r] + k];
                    e.val[idx] = (float)c.val[c.start[r] + k];
                } else {
                    e.col[idx] = r < rows ? r : 0;
                    e.val[idx] = 0.f;
                }
            }
            e.nnz += len;
        }
    }
    return e;
}

// ---------------------------------------------------------------------------
// Row tiles for the two-sweep Jacobi kernel: spatially compact groups of own
// rows (consecutive in the Morton order of the rest positions) and their halo
// (the other rows their off-diagonal entries reach).  Phase 1 of a launch
// computes one sweep for own + halo rows from global x into shared memory,
// phase 2 the next sweep for the own rows from shared memory.  Each tile's rows
// are padded to whole ELL slices so that no slice straddles two tiles.
// ---------------------------------------------------------------------------
struct HostTiles {
    int lanes = 1, ntiles = 0, max_local = 0;
    std::vector<int> row0, nlocal, nown, s1_0, s1_n, s2_0, s2_n;  // per tile
    std::vector<int> trow;                                        // local row -> global row (-1 = padding)
    HostEll e1, e2;                                               // phase 1 (global cols), phase 2 (local cols)
};

// Sliced ELL of explicit rows: rows[k] = (columns, values); padding column pad[k].
inline HostEll rows_to_sliced_ell(const std::vector<std::vector<int>>& cols, const std::vector<std::vector<double>>& vals,
                                  const std::vector<int>& pad, int T) {
    HostCsr c;
    const int rows = (int)cols.size();
    c.start.assign(rows + 1, 0);
    for (int r = 0; r < rows; r++) {
        c.start[r + 1] = c.start[r] + (int)cols[r].size();
        c.col.insert(c.col.end(), cols[r].begin(), cols[r].end());
        c.val.insert(c.val.end(), vals[r].begin(), vals[r].end());
    }
    HostEll e = csr_to_sliced_ell(c, rows, T);
    const int S = 32 / T;
    for (int sl = 0; sl < e.nslices; sl++) {  // padding entries: the row's own (valid) column
        const int w = (e.ptr[sl + 1] - e.ptr[sl]) / S;
        for (int lr = 0; lr < S; lr++) {
            const int r = sl * S + lr;
            const int len = r < rows ? (int)cols[r].size() : 0;
            for (int k = len; k < w; k++) e.col[e.ptr[sl] + (k / T) * 32 + (k % T) * S + lr] = r < rows ? pad[r] : pad[0];
        }
    }
    return e;
}

inline uint32_t spread10_host(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Tiles of `own` rows of the nd x nd off-diagonal CSR A (columns sorted), in the
// Morton order of the positions pos (xyz per row).
inline HostTiles build_tiles(const HostCsr& A, int nd, const float* pos, int pos_stride, int own, int T) {
    HostTiles t;
    t.lanes = T;
    const int S = 32 / T;
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < nd; i++)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], pos[pos_stride * i + k]);
            hi[k] = std::max(hi[k], pos[pos_stride * i + k]);
        }
    std::vector<std::pair<uint32_t, int>> key(nd);
    for (int i = 0; i < nd; i++) {
        uint32_t q[3];
        for (int k = 0; k < 3; k++) {
            const float ext = hi[k] - lo[k];
            const float u = ext > 0.f ? (pos[pos_stride * i + k] - lo[k]) / ext : 0.f;
            q[k] = (uint32_t)std::min(1023.f, std::max(0.f, u * 1023.f));
        }
        key[i] = {spread10_host(q[0]) | (spread10_host(q[1]) << 1) | (spread10_host(q[2]) << 2), i};
    }
    std::stable_sort(key.begin(), key.end());
    std::vector<int> local_of(nd, -1);
    std::vector<std::vector<int>> c1, c2;
    std::vector<std::vector<double>> v1, v2;
    std::vector<int> pad1, pad2;
    for (int b = 0; b < nd; b += own) {
        const int e = std::min(nd, b + own);
        std::vector<int> rows;
        for (int k = b; k < e; k++) rows.push_back(key[k].second);
        std::vector<int> halo;
        for (int r : rows) local_of[r] = -2;  // mark own
        for (int r : rows)
            for (int a = A.start[r]; a < A.start[r + 1]; a++)
                if (local_of[A.col[a]] == -1) {
                    local_of[A.col[a]] = -3;
                    halo.push_back(A.col[a]);
                }
        std::sort(halo.begin(), halo.end());
        std::vector<int> loc(rows);
        loc.insert(loc.end(), halo.begin(), halo.end());
        for (int k = 0; k < (int)loc.size(); k++) local_of[loc[k]] = k;
        const int n1 = (int)loc.size(), n1p = (n1 + S - 1) / S * S, nop = ((int)rows.size() + S - 1) / S * S;
        t.row0.push_back((int)t.trow.size());
        t.nlocal.push_back(n1);
        t.nown.push_back((int)rows.size());
        t.s1_0.push_back((int)c1.size() / S);
        t.s1_n.push_back(n1p / S);
        t.s2_0.push_back((int)c2.size() / S);
        t.s2_n.push_back(nop / S);
        t.max_local = std::max(t.max_local, n1p);
        for (int k = 0; k < n1p; k++) {
            const int g = k < n1 ? loc[k] : -1;
            t.trow.push_back(g);
            std::vector<int> cc;
            std::vector<double> vv;
            if (g >= 0)
                for (int a = A.start[g]; a < A.start[g + 1]; a++) {
                    cc.push_back(A.col[a]);
                    vv.push_back(A.val[a]);
                }
            c1.push_back(cc);
            v1.push_back(vv);
            pad1.push_back(g >= 0 ? g : loc[0]);
        }
        for (int k = 0; k < nop; k++) {
            std::vector<int> cc;
            std::vector<double> vv;
            if (k < (int)rows.size()) {
                const int g = rows[k];
                for (int a = A.start[g]; a < A.start[g + 1]; a++) {
                    cc.push_back(local_of[A.col[a]]);
                    vv.push_back(A.val[a]);
                }
            }
            c2.push_back(cc);
            v2.push_back(vv);
            pad2.push_back(k < (int)rows.size() ? k : 0);
        }
        for (int r : loc) local_of[r] = -1;
    }
    t.ntiles = (int)t.row0.size();
    t.e1 = rows_to_sliced_ell(c1, v1, pad1, T);
    t.e2 = rows_to_sliced_ell(c2, v2, pad2, T);
    return t;
}

struct Assembly {
    std::vector<float> a_diag;      // [nd]
    HostCsr A;                      // off-diagonal part, nd x nd (columns sorted)
    HostCsr R;                      // h^2 D^T W^2, nd x m (columns sorted)
    std::vector<float> wrow;        // [m]
    std::vector<float> dt2wc;       // [nd]
    int64_t nnz_D = 0;
    // backend_semantics 1: the CPU backend's damping matrix (added to A as well),
    // off-diagonal CSR and diagonal, for b_ini = Damp x0
    HostCsr damp;
    std::vector<float> damp_diag;
};

// Validates the description and assembles the constant matrices.  Returns an
// empty string on success, else the reason.
inline std::string assemble(const AdmmB200Desc& d, Assembly& out) {
    const int n = d.n_vert, nd = d.n_dyn, m = d.n_rows;
    if (n <= 0 || nd <= 0 || nd > n || m <= 0) return "n_vert/n_dyn/n_rows";
    auto chk_rows = [&](int sr, int cnt, int per) { return cnt == 0 || (sr >= 0 && sr + cnt * per <= m); };
    if (!chk_rows(d.tri_start_row, d.n_tri, 2) || !chk_rows(d.tet_start_row, d.n_tet, 3) ||
        !chk_rows(d.bend_start_row, d.n_bend, 1) || !chk_rows(d.pin_start_row, d.n_pin, 1))
        return "constraint rows exceed n_rows";
    std::vector<std::vector<std::pair<int, double>>> rows(m);
    std::vector<double> w(m, 0.0);
    auto vcheck = [&](int v) { return v >= 0 && v < nd; };
    for (int c = 0; c < d.n_tri; c++) {
        const int* id = d.tri_inds + 3 * c;
        const float* B = d.tri_binv + 4 * c;
        for (int k = 0; k < 3; k++) if (!vcheck(id[k])) return "tri_inds out of the dynamic range";
        for (int r = 0; r < 2; r++) {
            const double g0 = -((double)B[0 * 2 + r] + (double)B[1 * 2 + r]);
            const int row = d.tri_start_row + 2 * c + r;
            rows[row] = {{id[0], g0}, {id[1], (double)B[0 * 2 + r]}, {id[2], (double)B[1 * 2 + r]}};
            w[row] = d.tri_w[c];
        }
    }
    for (int c = 0; c < d.n_tet; c++) {
        const int* id = d.tet_inds + 4 * c;
        const float* B = d.tet_binv + 9 * c;
        for (int k = 0; k < 4; k++) if (!vcheck(id[k])) return "tet_inds out of the dynamic range";
        for (int r = 0; r < 3; r++) {
            const double g0 = -(((double)B[0 * 3 + r] + (double)B[1 * 3 + r]) + (double)B[2 * 3 + r]);
            const int row = d.tet_start_row + 3 * c + r;
            rows[row] = {{id[0], g0}, {id[1], (double)B[0 * 3 + r]}, {id[2], (double)B[1 * 3 + r]},
                         {id[3], (double)B[2 * 3 + r]}};
            w[row] = d.tet_w[c];
        }
    }
    for (int c = 0; c < d.n_bend; c++) {
        const int row = d.bend_start_row + c;
        if (d.bend_offsets[c + 1] < d.bend_offsets[c]) return "bend_offsets not increasing";
        for (int k = d.bend_offsets[c]; k < d.bend_offsets[c + 1]; k++) {
            if (!vcheck(d.bend_inds[k])) return "bend_inds out of the dynamic range";
            rows[row].push_back({d.bend_inds[k], (double)d.bend_coeffs[k]});
        }
        w[row] = d.bend_w[c];
    }
    for (int c = 0; c < d.n_pin; c++) {
        if (!vcheck(d.pin_inds[c])) return "pin_inds out of the dynamic range";
        const int row = d.pin_start_row + c;
        rows[row] = {{d.pin_inds[c], 1.0}};
        w[row] = d.pin_w[c];
    }
    const double h2 = (double)d.dt * (double)d.dt;
    // sum duplicate columns within a row (Eigen setFromTriplets)
    for (auto& r : rows) {
        std::sort(r.begin(), r.end(), [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
            return a.first < b.first;
        });
        std::vector<std::pair<int, double>> u;
        for (auto& e : r) {
            if (!u.empty() && u.back().first == e.first) u.back().second += e.second;
            else u.push_back(e);
        }
        r.swap(u);
        out.nnz_D += (int64_t)r.size();
    }
    std::vector<std::unordered_map<int, double>> arow(nd);
    std::vector<std::vector<std::pair<int, double>>> rt(nd);
    for (int r = 0; r < m; r++) {
        const double w2 = w[r] * w[r] * h2;
        for (auto& a : rows[r]) {
            rt[a.first].push_back({r, w2 * a.second});
            for (auto& b : rows[r]) arow[a.first][b.first] += w2 * a.second * b.second;
        }
    }
    // Rayleigh damping of the CPU backend (admm_impl_cpu.cpp:181-191):
    // Damp = dt (damp_k_L Dd^T Wd Dd + damp_k_M M) over the triangle, tet and bending
    // rows (constraint types below 4), Wd = diag(w); A_damp = A + Damp (:221).
    std::vector<std::unordered_map<int, double>> drow;
    if (d.backend_semantics == 1) {
        drow.resize(nd);
        const double kL = (double)d.damp_k_L, kM = (double)d.damp_k_M, h = (double)d.dt;
        auto damped = [&](int r) {
            return (d.n_tri && r >= d.tri_start_row && r < d.tri_start_row + 2 * d.n_tri) ||
                   (d.n_tet && r >= d.tet_start_row && r < d.tet_start_row + 3 * d.n_tet) ||
                   (d.n_bend && r >= d.bend_start_row && r < d.bend_start_row + d.n_bend);
        };
        for (int r = 0; r < m; r++) {
            if (!damped(r)) continue;
            const double s = h * kL * w[r];
            for (auto& a : rows[r])
                for (auto& b : rows[r]) drow[a.first][b.first] += s * a.second * b.second;
        }
        for (int i = 0; i < nd; i++) drow[i][i] += h * kM * (double)d.mass[i];
        for (int i = 0; i < nd; i++)
            for (auto& kv : drow[i]) arow[i][kv.first] += kv.second;
    }
    out.dt2wc.assign(nd, 0.f);
    if (d.enable_contact) {
        std::vector<char> surf(n, 0);
        for (int k = 0; k < d.n_surf_vert; k++) {
            const int v = d.surf_verts[k];
            if (v < 0 || v >= n) return "surf_verts out of range";
            surf[v] = 1;
        }
        for (int i = 0; i < nd; i++)
            if (surf[i]) out.dt2wc[i] = (float)(h2 * (double)d.contact_w[i]);
    }
    HostCsr ac, rc;
    ac.start.assign(nd + 1, 0);
    rc.start.assign(nd + 1, 0);
    out.a_diag.assign(nd, 0.f);
    for (int i = 0; i < nd; i++) {
        std::vector<std::pair<int, double>> e(arow[i].begin(), arow[i].end());
        std::sort(e.begin(), e.end());
        double diag = (double)d.mass[i] + (d.enable_contact ? (double)out.dt2wc[i] : 0.0);
        for (auto& kv : e) {
            if (kv.first == i) diag += kv.second;
            else { ac.col.push_back(kv.first); ac.val.push_back(kv.second); }
        }
        if (!(diag > 0.0)) return "non-positive diagonal in the system matrix";
        out.a_diag[i] = (float)diag;
        ac.start[i + 1] = (int)ac.col.size();
        std::sort(rt[i].begin(), rt[i].end());
        for (auto& kv : rt[i]) { rc.col.push_back(kv.first); rc.val.push_back(kv.second); }
        rc.start[i + 1] = (int)rc.col.size();
    }
    if (d.backend_semantics == 1) {
        HostCsr dc;
        dc.start.assign(nd + 1, 0);
        out.damp_diag.assign(nd, 0.f);
        for (int i = 0; i < nd; i++) {
            std::vector<std::pair<int, double>> e(drow[i].begin(), drow[i].end());
            std::sort(e.begin(), e.end());
            for (auto& kv : e) {
                if (kv.first == i) out.damp_diag[i] = (float)kv.second;
                else { dc.col.push_back(kv.first); dc.val.push_back(kv.second); }
            }
            dc.start[i + 1] = (int)dc.col.size();
        }
        out.damp = std::move(dc);
    }
    out.A = std::move(ac);
    out.R = std::move(rc);
    out.wrow.assign(m, 0.f);
    for (int r = 0; r < m; r++) out.wrow[r] = (float)w[r];
    return "";
}

}  // namespace admm
