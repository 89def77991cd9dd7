// Checks of the sliced-ELL layout built on the host (parallel_admm_b200/csrc/setup.hpp),
// against a CSR matrix, by emulating in C++ what the row-sum kernels do on the GPU
// (kernels.cuh: ell_row_sum / EllRowPf): lane l of the warp of slice w takes the entries
// ptr[w] + l + 32 j in order j = 0, 1, ... with fmaf, then the lanes of a row are combined
// by xor shuffles with offsets S, 2S, ..., 16 (S = 32 / T rows per slice).
//
//  1. every slot maps to a row (rowid is a permutation of each 32-row window; slots past the
//     last row hold `rows`), every row's entries appear once with their values;
//  2. the emulated row sums equal a CSR product exactly for integer-valued data;
//  3. the row-order permutation does not change any row's bits (same entries, same order,
//     same lane layout; only the slot and the padding differ);
//  4. on rows that alternate between 6 and 18 entries the permutation shrinks the padding
//     when a slice holds fewer rows than a window (T > 1).
// Exit code 0 on success; a message on stderr and exit code 1 otherwise.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "setup.hpp"

using admm::HostCsr;
using admm::HostEll;

static int g_fail = 0;
#define CHECK(cond, ...)                          \
    do {                                          \
        if (!(cond)) {                            \
            std::fprintf(stderr, __VA_ARGS__);    \
            std::fprintf(stderr, "\n");           \
            g_fail = 1;                           \
            return;                               \
        }                                         \
    } while (0)

struct V3 {
    float x, y, z;
};

static HostCsr random_csr(int rows, int max_len, bool integers, std::mt19937& rng, bool alternate = false) {
    HostCsr c;
    c.start.assign(rows + 1, 0);
    std::uniform_int_distribution<int> len_d(0, max_len), col_d(0, rows - 1), ival(-4, 4);
    std::uniform_real_distribution<double> rval(-1.0, 1.0);
    for (int r = 0; r < rows; r++) {
        const int len = alternate ? (r % 2 ? 18 : 6) : len_d(rng);
        for (int k = 0; k < len; k++) {
            c.col.push_back(col_d(rng));
            c.val.push_back(integers ? (double)ival(rng) : rval(rng));
        }
        c.start[r + 1] = (int)c.col.size();
    }
    return c;
}

// Row sums as the kernel computes them; out[r] for every row r.
static std::vector<V3> emulate(const HostEll& e, const std::vector<V3>& v) {
    const int T = e.lanes, S = 32 / T;
    std::vector<V3> out(e.rows, V3{0.f, 0.f, 0.f});
    for (int w = 0; w < e.nslices; w++) {
        V3 acc[32];
        const int b = e.ptr[w], end = e.ptr[w + 1];
        for (int l = 0; l < 32; l++) {
            float ax = 0.f, ay = 0.f, az = 0.f;
            for (int k = b + l; k < end; k += 32) {
                const V3 q = v[e.col[k]];
                const float a = e.val[k];
                ax = std::fma(a, q.x, ax);
                ay = std::fma(a, q.y, ay);
                az = std::fma(a, q.z, az);
            }
            acc[l] = V3{ax, ay, az};
        }
        for (int o = S; o < 32; o <<= 1) {
            V3 nxt[32];
            for (int l = 0; l < 32; l++)
                nxt[l] = V3{acc[l].x + acc[l ^ o].x, acc[l].y + acc[l ^ o].y, acc[l].z + acc[l ^ o].z};
            for (int l = 0; l < 32; l++) acc[l] = nxt[l];
        }
        for (int lr = 0; lr < S; lr++) {
            const int slot = w * S + lr;
            const int r = e.rowid.empty() ? slot : e.rowid[slot];
            if (r < e.rows) out[r] = acc[lr];
        }
    }
    return out;
}

static void check_layout(const HostCsr& c, const HostEll& e, bool permute) {
    const int T = e.lanes, S = 32 / T, rows = e.rows;
    CHECK((int)e.ptr.size() == e.nslices + 1, "ptr size");
    CHECK(e.nslices == (rows + S - 1) / S, "slice count");
    if (permute) {
        CHECK((int)e.rowid.size() == e.nslices * S, "rowid size %zu", e.rowid.size());
        for (int w0 = 0; w0 < e.nslices * S; w0 += 32) {
            std::vector<int> seen;
            for (int k = w0; k < std::min(w0 + 32, e.nslices * S); k++) {
                const int r = e.rowid[k];
                if (k >= rows) {
                    CHECK(r == rows, "slot %d past the last row maps to %d", k, r);
                    continue;
                }
                CHECK(r >= w0 && r < std::min(w0 + 32, rows), "slot %d maps to row %d outside its window", k, r);
                seen.push_back(r);
            }
            std::sort(seen.begin(), seen.end());
            for (size_t i = 0; i < seen.size(); i++) CHECK(seen[i] == w0 + (int)i, "window %d is not a permutation", w0);
        }
    } else {
        CHECK(e.rowid.empty(), "rowid without permutation");
    }
    // every row's entries, in order, at (k / T) * 32 + (k % T) * S + slot
    int64_t nnz = 0;
    for (int w = 0; w < e.nslices; w++) {
        const int width = (e.ptr[w + 1] - e.ptr[w]) / S;
        CHECK(width % T == 0, "slice %d width %d not a multiple of T", w, width);
        for (int lr = 0; lr < S; lr++) {
            const int slot = w * S + lr;
            const int r = e.rowid.empty() ? slot : e.rowid[slot];
            const int len = r < rows ? c.start[r + 1] - c.start[r] : 0;
            CHECK(len <= width, "row %d longer than its slice", r);
            for (int k = 0; k < width; k++) {
                const int idx = e.ptr[w] + (k / T) * 32 + (k % T) * S + lr;
                if (k < len) {
                    CHECK(e.col[idx] == c.col[c.start[r] + k] && e.val[idx] == (float)c.val[c.start[r] + k],
                          "row %d entry %d misplaced", r, k);
                } else {
                    CHECK(e.val[idx] == 0.f && e.col[idx] >= 0 && e.col[idx] < std::max(rows, 1),
                          "padding of row %d not a zero entry on a valid column", r);
                }
            }
            nnz += len;
        }
    }
    CHECK(nnz == e.nnz && nnz == (int64_t)c.col.size(), "entry count %lld vs %zu", (long long)nnz, c.col.size());
}

static void run_case(int rows, int max_len, int T, uint32_t seed) {
    std::mt19937 rng(seed);
    // integer data: every sum is exact, so the emulated kernel equals the CSR product
    {
        const HostCsr c = random_csr(rows, max_len, true, rng);
        std::vector<V3> v(rows);
        std::uniform_int_distribution<int> d(-8, 8);
        for (auto& q : v) q = V3{(float)d(rng), (float)d(rng), (float)d(rng)};
        for (int permute = 0; permute < 2; permute++) {
            const HostEll e = admm::csr_to_sliced_ell(c, rows, T, permute != 0);
            check_layout(c, e, permute != 0);
            if (g_fail) return;
            const std::vector<V3> y = emulate(e, v);
            for (int r = 0; r < rows; r++) {
                double sx = 0, sy = 0, sz = 0;
                for (int k = c.start[r]; k < c.start[r + 1]; k++) {
                    sx += c.val[k] * v[c.col[k]].x;
                    sy += c.val[k] * v[c.col[k]].y;
                    sz += c.val[k] * v[c.col[k]].z;
                }
                CHECK(y[r].x == (float)sx && y[r].y == (float)sy && y[r].z == (float)sz,
                      "rows=%d T=%d permute=%d row %d: %g vs %g", rows, T, permute, r, y[r].x, sx);
            }
        }
    }
    // real data: the permuted layout gives the same bits as the plain one, row by row
    {
        const HostCsr c = random_csr(rows, max_len, false, rng);
        std::vector<V3> v(rows);
        std::uniform_real_distribution<float> d(-2.f, 2.f);
        for (auto& q : v) q = V3{d(rng), d(rng), d(rng)};
        const std::vector<V3> a = emulate(admm::csr_to_sliced_ell(c, rows, T, false), v);
        const std::vector<V3> b = emulate(admm::csr_to_sliced_ell(c, rows, T, true), v);
        for (int r = 0; r < rows; r++)
            CHECK(std::memcmp(&a[r], &b[r], sizeof(V3)) == 0, "rows=%d T=%d row %d: permuted sum differs", rows, T, r);
    }
}

int main() {
    const int sizes[] = {1, 31, 32, 33, 100, 1000};
    const int lanes[] = {1, 2, 4, 8};
    uint32_t seed = 1;
    for (int rows : sizes)
        for (int T : lanes)
            for (int max_len : {0, 5, 40, 300}) {
                run_case(rows, max_len, T, seed++);
                if (g_fail) return 1;
            }
    // a tet lattice's alternating 6 / 18 neighbours: the permutation cuts the padding
    std::mt19937 rng(7);
    const HostCsr c = random_csr(4096, 0, false, rng, true);
    for (int T : lanes) {
        const HostEll plain = admm::csr_to_sliced_ell(c, 4096, T, false);
        const HostEll perm = admm::csr_to_sliced_ell(c, 4096, T, true);
        const double pad_plain = (double)plain.ptr.back() / plain.nnz - 1.0;
        const double pad_perm = (double)perm.ptr.back() / perm.nnz - 1.0;
        std::printf("T=%d padding plain %.3f permuted %.3f\n", T, pad_plain, pad_perm);
        // T = 1: a slice is the whole 32-row window, whose width no order changes
        if (T == 1 ? pad_perm != pad_plain : !(pad_perm < pad_plain)) {
            std::fprintf(stderr, "T=%d: padding %.3f with the permutation, %.3f without\n", T, pad_perm, pad_plain);
            return 1;
        }
    }
    std::printf("ok\n");
    return 0;
}
