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
inline HostEll csr_to_sliced_ell(const HostCsr& c, int rows, int T) {
    HostEll e;
    const int S = 32 / T;
    e.rows = rows;
    e.lanes = T;
    e.nslices = (rows + S - 1) / S;
    e.ptr.assign(e.nslices + 1, 0);
    for (int s = 0; s < e.nslices; s++) {
        int w = 0;
        for (int r = s * S; r < std::min(rows, (s + 1) * S); r++) w = std::max(w, c.start[r + 1] - c.start[r]);
        w = (w + T - 1) / T * T;
        e.ptr[s + 1] = e.ptr[s] + w * S;
    }
    e.col.assign(e.ptr[e.nslices], 0);
    e.val.assign(e.ptr[e.nslices], 0.f);
    for (int s = 0; s < e.nslices; s++) {
        const int w = (e.ptr[s + 1] - e.ptr[s]) / S;
        for (int lr = 0; lr < S; lr++) {
            const int r = s * S + lr;
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

struct Assembly {
    std::vector<float> a_diag;      // [nd]
    HostCsr A;                      // off-diagonal part, nd x nd (columns sorted)
    HostCsr R;                      // h^2 D^T W^2, nd x m (columns sorted)
    std::vector<float> wrow;        // [m]
    std::vector<float> dt2wc;       // [nd]
    int64_t nnz_D = 0;
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
    out.A = std::move(ac);
    out.R = std::move(rc);
    out.wrow.assign(m, 0.f);
    for (int r = 0; r < m; r++) out.wrow[r] = (float)w[r];
    return "";
}

}  // namespace admm
