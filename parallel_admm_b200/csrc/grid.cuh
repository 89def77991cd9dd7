// grid.cuh -- uniform-grid (spatial hash) broad phase for the DCD.
//
// The contact pair set of the reference's DCD (lbvh.cu:1693-1813) does not
// depend on the acceleration structure: a pair is reported when the query box
// overlaps the element box under the reference's rule (lbvh.cu:43-49) and the
// region-0 narrow phase accepts it.  A BVH query is a chain of dependent node
// loads (tens of L2 round trips per query for a few thousand queries, far too
// few threads to hide them); a grid query issues the loads of all of its cells
// at once, so a DCD costs a handful of round trips.
//
// Layout: every surface triangle and edge whose box spans at most kGridMaxSpan
// cells per axis is inserted into each cell it overlaps, in a hash table of
// (cell, type) buckets built by count -> scan -> scatter; each entry carries
// the element's box, so that the box test needs no further load.  Larger
// elements (and any that do not fit the entry capacity) go to a per-type "big"
// list that the queries scan directly.
//
// Each pair is reported once: a query visits the cells of its box inflated by
// the gap (plus a margin that covers the rounding of the overlap test), and
// accepts an element only in the cell that is the lower corner of the overlap
// of the two cell ranges.  Edge-edge pairs (a, b), a < b, with both edges in the
// grid belong to a; a pair of one grid edge and one big edge belongs to the
// grid edge; a pair of two big edges to the smaller index.  Every query sorts
// its output segment by partner index, so the contact list is independent of
// atomic arrival order.
#pragma once
#include "common.cuh"
#include "lbvh.cuh"
#include "scene_dev.cuh"

namespace admm {

constexpr int kGridMaxSpan = 4;  // cells per axis an element may span in the grid

ADMM_DEV int grid_cell(float v, float inv_c) {
    float f = floorf(v * inv_c);
    f = fminf(fmaxf(f, -1073741824.f), 1073741824.f);
    return (int)f;
}

ADMM_DEV int grid_bucket(int ix, int iy, int iz, int type, int hmask) {
    const unsigned h = ((unsigned)ix * 73856093u) ^ ((unsigned)iy * 19349663u) ^ ((unsigned)iz * 83492791u) ^
                       ((unsigned)type * 2654435761u);
    return (int)(h & (unsigned)hmask);
}

// Box of surface element u (triangles first, then edges); type 0 = triangle.
ADMM_DEV void grid_elem_box(const DevScene& s, int u, int& type, int& id, float4& lo, float4& up) {
    lo = f4(1e32f, 1e32f, 1e32f);
    up = f4(-1e32f, -1e32f, -1e32f);
    if (u < s.nst) {
        type = 0;
        id = u;
        const int4 t = s.st[u];
        box_add(lo, up, s.x[t.x]);
        box_add(lo, up, s.x[t.y]);
        box_add(lo, up, s.x[t.z]);
    } else {
        type = 1;
        id = u - s.nst;
        const int2 e = s.se[id];
        box_add(lo, up, s.x[e.x]);
        box_add(lo, up, s.x[e.y]);
    }
}

ADMM_DEV void grid_range(const float4& lo, const float4& up, float inv_c, int3& a, int3& b) {
    a = make_int3(grid_cell(lo.x, inv_c), grid_cell(lo.y, inv_c), grid_cell(lo.z, inv_c));
    b = make_int3(grid_cell(up.x, inv_c), grid_cell(up.y, inv_c), grid_cell(up.z, inv_c));
}

// Cell range of a query box inflated by the gap.  The margin keeps every element
// that passes box_overlap inside the range despite the rounding of its
// subtractions (a few ulps of the coordinates).
ADMM_DEV float grid_pad(float v, float gap) { return gap + fmaxf(gap, fabsf(v)) * (1.f / 1048576.f); }

// A query whose cell range is larger than this (a stretched element or far-out
// coordinates) tests every grid element of the type directly instead.
constexpr int kGridMaxQueryCells = 512;

ADMM_DEV bool grid_range_small(int3 a, int3 b) {
    const long long n = (long long)(b.x - a.x + 1) * (long long)(b.y - a.y + 1) * (long long)(b.z - a.z + 1);
    return n >= 1 && n <= kGridMaxQueryCells;
}

ADMM_DEV void grid_query_range(const float4& lo, const float4& up, float gap, float inv_c, int3& a, int3& b) {
    a = make_int3(grid_cell(lo.x - grid_pad(lo.x, gap), inv_c), grid_cell(lo.y - grid_pad(lo.y, gap), inv_c),
                  grid_cell(lo.z - grid_pad(lo.z, gap), inv_c));
    b = make_int3(grid_cell(up.x + grid_pad(up.x, gap), inv_c), grid_cell(up.y + grid_pad(up.y, gap), inv_c),
                  grid_cell(up.z + grid_pad(up.z, gap), inv_c));
}

// Calls f(bucket) once for every distinct bucket of the cells [a, b] of one
// element (two cells of an element may hash to the same bucket; the element is
// entered there once).  Spans are at most kGridMaxSpan per axis.
template <class F>
ADMM_DEV void grid_for_buckets(int3 a, int3 b, int type, int hmask, F f) {
    int seen[kGridMaxSpan * kGridMaxSpan * kGridMaxSpan];
    int ns = 0;
    for (int iz = a.z; iz <= b.z; iz++)
        for (int iy = a.y; iy <= b.y; iy++)
            for (int ix = a.x; ix <= b.x; ix++) {
                const int bk = grid_bucket(ix, iy, iz, type, hmask);
                bool dup = false;
                for (int j = 0; j < ns; j++) dup |= seen[j] == bk;
                if (!dup) {
                    seen[ns++] = bk;
                    f(bk);
                }
            }
}

// Pass 1: bucket counts; elements that are too large (or beyond the entry
// capacity) go to the big lists.  ctr[0] = entries reserved, ctr[1..2] = big
// triangle / edge counts (zeroed before the launch).
__global__ void __launch_bounds__(256) k_grid_count(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const GridDev& g = s.grid;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= s.nst + s.nse) return;
    int type, id;
    float4 lo, up;
    grid_elem_box(s, u, type, id, lo, up);
    int3 a, b;
    grid_range(lo, up, g.inv_c, a, b);
    const int sx = b.x - a.x + 1, sy = b.y - a.y + 1, sz = b.z - a.z + 1;
    bool in_grid = sx >= 1 && sy >= 1 && sz >= 1 && sx <= kGridMaxSpan && sy <= kGridMaxSpan && sz <= kGridMaxSpan;
    if (in_grid) {
        const int nc = sx * sy * sz;
        const int r = atomicAdd(&g.ctr[0], nc);
        in_grid = r + nc <= g.cap;
    }
    g.mode[u] = in_grid ? 1 : 0;
    if (in_grid) {
        grid_for_buckets(a, b, type, g.hmask, [&](int bk) { atomicAdd(&g.cnt[bk], 1); });
    } else {
        const int k = atomicAdd(&g.ctr[1 + type], 1);
        (type == 0 ? g.big_tri : g.big_edge)[k] = id;
    }
}

// Pass 2 (after the scan of the counts into start): entries, one per element
// and cell; the counts are consumed back to zero for the next DCD.
__global__ void __launch_bounds__(256) k_grid_scatter(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const GridDev& g = s.grid;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= s.nst + s.nse || !g.mode[u]) return;
    int type, id;
    float4 lo, up;
    grid_elem_box(s, u, type, id, lo, up);
    int3 a, b;
    grid_range(lo, up, g.inv_c, a, b);
    lo.w = __int_as_float(id);
    up.w = __int_as_float(type);
    grid_for_buckets(a, b, type, g.hmask, [&](int bk) {
        const int pos = g.start[bk] + atomicSub(&g.cnt[bk], 1) - 1;
        g.ent_lo[pos] = lo;
        g.ent_up[pos] = up;
    });
}

// One accepted pair: count it, or (WRITE) store it at slot base + count.
template <bool WRITE>
ADMM_DEV void grid_emit(const DevScene& s, int base, int& count, int partner, int4 ids, const NpResult& r, bool ee) {
    if (WRITE) {
        const int slot = base + count;
        if (slot < s.cap) {
            write_contact(s, slot, ids, r, ee);
            s.grid.qkey[slot] = partner;
        }
    }
    count++;
}

// Insertion sort of the slots [b, e) by partner index (all contact arrays).
ADMM_DEV void grid_sort_segment(const DevScene& s, int b, int e) {
    int* key = s.grid.qkey;
    for (int k = b + 1; k < e; k++) {
        const int kk = key[k];
        const int4 pr = s.pairs[k];
        const float4 pt = s.point[k], ba = s.bary[k], nr = s.nrm[k];
        int j = k - 1;
        while (j >= b && key[j] > kk) {
            key[j + 1] = key[j];
            s.pairs[j + 1] = s.pairs[j];
            s.point[j + 1] = s.point[j];
            s.bary[j + 1] = s.bary[j];
            s.nrm[j + 1] = s.nrm[j];
            j--;
        }
        key[j + 1] = kk;
        s.pairs[j + 1] = pr;
        s.point[j + 1] = pt;
        s.bary[j + 1] = ba;
        s.nrm[j + 1] = nr;
    }
}

// Vertex-face query of surface vertex q (lbvh.cu:1693-1748 semantics).
template <bool WRITE>
ADMM_DEV int grid_query_vf(const DevScene& s, int q, int base) {
    const GridDev& g = s.grid;
    const int v = s.sv[q];
    const float4 P = s.x[v];
    const float gap = s.thickness;
    int count = 0;
    auto test = [&](int f) {
        const int4 tri = s.st[f];
        if (v == tri.x || v == tri.y || v == tri.z) return;
        NpResult r;
        if (narrow_pt(P, s.x[tri.x], s.x[tri.y], s.x[tri.z], r) && r.dist < gap && r.dist >= 0.f)
            grid_emit<WRITE>(s, base, count, f, make_int4(v, tri.x, tri.y, tri.z), r, false);
    };
    int3 a, b;
    grid_query_range(P, P, gap, g.inv_c, a, b);
    if (grid_range_small(a, b)) {
        for (int iz = a.z; iz <= b.z; iz++)
            for (int iy = a.y; iy <= b.y; iy++)
                for (int ix = a.x; ix <= b.x; ix++) {
                    const int bk = grid_bucket(ix, iy, iz, 0, g.hmask);
                    const int k1 = g.start[bk + 1];
                    for (int k = g.start[bk]; k < k1; k++) {
                        const float4 lo = g.ent_lo[k], up = g.ent_up[k];
                        if (__float_as_int(up.w) != 0 || !box_overlap(P, P, lo, up, gap)) continue;
                        int3 ea, eb;
                        grid_range(lo, up, g.inv_c, ea, eb);
                        if (max(a.x, ea.x) != ix || max(a.y, ea.y) != iy || max(a.z, ea.z) != iz) continue;
                        test(__float_as_int(lo.w));
                    }
                }
    } else {
        for (int f = 0; f < s.nst; f++) {
            if (!g.mode[f]) continue;
            const int4 tri = s.st[f];
            float4 lo = f4(1e32f, 1e32f, 1e32f), up = f4(-1e32f, -1e32f, -1e32f);
            box_add(lo, up, s.x[tri.x]);
            box_add(lo, up, s.x[tri.y]);
            box_add(lo, up, s.x[tri.z]);
            if (box_overlap(P, P, lo, up, gap)) test(f);
        }
    }
    const int nb = g.ctr[1];
    for (int j = 0; j < nb; j++) {
        const int f = g.big_tri[j];
        const int4 tri = s.st[f];
        float4 lo = f4(1e32f, 1e32f, 1e32f), up = f4(-1e32f, -1e32f, -1e32f);
        box_add(lo, up, s.x[tri.x]);
        box_add(lo, up, s.x[tri.y]);
        box_add(lo, up, s.x[tri.z]);
        if (box_overlap(P, P, lo, up, gap)) test(f);
    }
    return count;
}

// Edge-edge query of surface edge e (lbvh.cu:1750-1813 semantics: pairs of
// edges that share no vertex, lower index first).
template <bool WRITE>
ADMM_DEV int grid_query_ee(const DevScene& s, int e, int base) {
    const GridDev& g = s.grid;
    const int2 ed = s.se[e];
    const float4 A0 = s.x[ed.x], A1 = s.x[ed.y];
    float4 lo = f4(1e32f, 1e32f, 1e32f), up = f4(-1e32f, -1e32f, -1e32f);
    box_add(lo, up, A0);
    box_add(lo, up, A1);
    const float gap = s.thickness;
    const bool small = g.mode[s.nst + e] != 0;
    int count = 0;
    auto test = [&](int o) {
        const int2 od = s.se[o];
        if (ed.x == od.x || ed.x == od.y || ed.y == od.x || ed.y == od.y) return;
        NpResult r;
        if (o > e) {
            if (narrow_ee(A0, A1, s.x[od.x], s.x[od.y], r) && r.dist < gap && r.dist >= 0.f)
                grid_emit<WRITE>(s, base, count, o, make_int4(ed.x, ed.y, od.x, od.y), r, true);
        } else {
            if (narrow_ee(s.x[od.x], s.x[od.y], A0, A1, r) && r.dist < gap && r.dist >= 0.f)
                grid_emit<WRITE>(s, base, count, o, make_int4(od.x, od.y, ed.x, ed.y), r, true);
        }
    };
    int3 a, b;
    grid_query_range(lo, up, gap, g.inv_c, a, b);
    if (small && !grid_range_small(a, b)) {
        for (int o = e + 1; o < s.nse; o++) {
            if (!g.mode[s.nst + o]) continue;
            const int2 od = s.se[o];
            float4 olo = f4(1e32f, 1e32f, 1e32f), oup = f4(-1e32f, -1e32f, -1e32f);
            box_add(olo, oup, s.x[od.x]);
            box_add(olo, oup, s.x[od.y]);
            if (box_overlap(lo, up, olo, oup, gap)) test(o);
        }
    } else if (small) {
        for (int iz = a.z; iz <= b.z; iz++)
            for (int iy = a.y; iy <= b.y; iy++)
                for (int ix = a.x; ix <= b.x; ix++) {
                    const int bk = grid_bucket(ix, iy, iz, 1, g.hmask);
                    const int k1 = g.start[bk + 1];
                    for (int k = g.start[bk]; k < k1; k++) {
                        const float4 elo = g.ent_lo[k], eup = g.ent_up[k];
                        const int o = __float_as_int(elo.w);
                        if (__float_as_int(eup.w) != 1 || o <= e || !box_overlap(lo, up, elo, eup, gap)) continue;
                        int3 ea, eb;
                        grid_range(elo, eup, g.inv_c, ea, eb);
                        if (max(a.x, ea.x) != ix || max(a.y, ea.y) != iy || max(a.z, ea.z) != iz) continue;
                        test(o);
                    }
                }
    }
    const int nb = g.ctr[2];
    for (int j = 0; j < nb; j++) {
        const int o = g.big_edge[j];
        // a grid edge owns its pairs with every big edge; two big edges: the lower index
        if (o == e || (!small && o < e)) continue;
        const int2 od = s.se[o];
        float4 olo = f4(1e32f, 1e32f, 1e32f), oup = f4(-1e32f, -1e32f, -1e32f);
        box_add(olo, oup, s.x[od.x]);
        box_add(olo, oup, s.x[od.y]);
        if (box_overlap(lo, up, olo, oup, gap)) test(o);  // the overlap rule is symmetric
    }
    return count;
}

// Count (WRITE = false: qcount) or write (WRITE = true, at qoff) the pairs of
// every query: surface vertices first, then surface edges.
template <bool WRITE>
__global__ void __launch_bounds__(128) k_grid_query(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= s.nsv + s.nse) return;
    const int base = WRITE ? s.qoff[q] : 0;
    const int n = q < s.nsv ? grid_query_vf<WRITE>(s, q, base) : grid_query_ee<WRITE>(s, q - s.nsv, base);
    if (!WRITE) {
        s.qcount[q] = n;
    } else {
        const int e = min(base + n, s.cap);
        if (e - base > 1) grid_sort_segment(s, base, e);
    }
}

}  // namespace admm
