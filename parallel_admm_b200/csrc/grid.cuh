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
// the element's box and the key of the cell it was entered for, so that other
// cells sharing the bucket are rejected by one 8-byte compare and the box test
// needs no further load.  Larger
// elements (and any that do not fit the entry capacity) go to a per-type "big"
// list that the queries scan directly.
//
// Each pair is reported once: a query visits the cells of its box inflated by
// the gap (plus a margin that covers the rounding of the overlap test), and
// accepts an element only in the cell that is the lower corner of the overlap
// of the two cell ranges -- the cell that, on every axis, is the first of the
// query's range or the first of the element's (entries carry the latter as
// three bits).  Edge-edge pairs (a, b), a < b, with both edges in the
// grid belong to a; a pair of one grid edge and one big edge belongs to the
// grid edge; a pair of two big edges to the smaller index.  Every query sorts
// its output segment by partner index, so the contact list is independent of
// atomic arrival order.
#pragma once
#include "common.cuh"
#include "lbvh.cuh"
#include "scene_dev.cuh"

namespace admm {

constexpr int kGridMaxSpan = 16;  // cells per axis an element may span in the grid

ADMM_DEV int grid_cell(float v, float inv_c) {
    float f = floorf(v * inv_c);
    f = fminf(fmaxf(f, -1048575.f), 1048575.f);  // the cell key holds 21 bits per coordinate
    return (int)f;
}

// Bucket of a cell: the low bits of the cell's Morton code, triangles in the
// lower half of the table, edges in the upper half.  Neighbouring cells land in
// neighbouring buckets, so the queries of neighbouring mesh vertices (which run
// in the same warps) read the same cache lines; cells whose codes differ only
// above the table size share a bucket and are told apart by the entry's cell key.
ADMM_DEV unsigned grid_spread10(unsigned v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

ADMM_DEV int grid_bucket(int ix, int iy, int iz, int type, int hmask) {
    const unsigned m = grid_spread10((unsigned)ix) | (grid_spread10((unsigned)iy) << 1) |
                       (grid_spread10((unsigned)iz) << 2);
    const unsigned half = (unsigned)hmask >> 1;  // hmask + 1 is a power of two >= 2
    return (int)((m & half) + (type ? half + 1u : 0u));
}

// 64-bit key of a cell (21 bits per coordinate, offset to non-negative).
ADMM_DEV unsigned long long grid_cell_key(int ix, int iy, int iz) {
    const unsigned long long o = 1ull << 20, m = (1ull << 21) - 1ull;
    return (((unsigned long long)(ix + (int)o) & m) << 42) | (((unsigned long long)(iy + (int)o) & m) << 21) |
           ((unsigned long long)(iz + (int)o) & m);
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
constexpr int kGridMaxQueryCells = 8192;

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

// Calls f(cell, bucket) for every cell [a, b] of one element.
template <class F>
ADMM_DEV void grid_for_cells(int3 a, int3 b, int type, int hmask, F f) {
    for (int iz = a.z; iz <= b.z; iz++)
        for (int iy = a.y; iy <= b.y; iy++)
            for (int ix = a.x; ix <= b.x; ix++) f(make_int4(ix, iy, iz, 0), grid_bucket(ix, iy, iz, type, hmask));
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
        grid_for_cells(a, b, type, g.hmask, [&](int4, int bk) { atomicAdd(&g.cnt[bk], 1); });
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
    grid_for_cells(a, b, type, g.hmask, [&](int4 c, int bk) {
        const int pos = g.start[bk] + atomicSub(&g.cnt[bk], 1) - 1;
        // w of up: for each axis, whether this cell is the element's first
        const int first = (c.x == a.x ? 1 : 0) | (c.y == a.y ? 2 : 0) | (c.z == a.z ? 4 : 0);
        g.ent_lo[pos] = lo;
        g.ent_up[pos] = make_float4(up.x, up.y, up.z, __int_as_float(first));
        g.ent_key[pos] = grid_cell_key(c.x, c.y, c.z);
    });
}

// Insertion sort of the contact slots [b, e) by partner index.
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

// ---------------------------------------------------------------------------
// Queries.  kQueryLanes consecutive threads serve one query: they split its
// cells (and the big lists) between them, so that the loads of different
// cells are in flight at the same time.  Each walk calls f(partner) for every
// element that passes the box test and the once-per-pair cell rule; f applies
// the index rules and the narrow phase.
// ---------------------------------------------------------------------------
constexpr int kQueryLanes = 8;
constexpr int kQueryHits = 4;  // hits per lane that the count pass records for the write pass

ADMM_DEV int3 grid_cell_at(int3 a, int3 b, int ci) {
    const int dx = b.x - a.x + 1, dy = b.y - a.y + 1;
    return make_int3(a.x + ci % dx, a.y + (ci / dx) % dy, a.z + ci / (dx * dy));
}

ADMM_DEV int grid_cells(int3 a, int3 b) { return (b.x - a.x + 1) * (b.y - a.y + 1) * (b.z - a.z + 1); }

ADMM_DEV float4 tri_box_lo(const DevScene& s, int f, float4& up) {
    const int4 t = s.st[f];
    float4 lo = f4(1e32f, 1e32f, 1e32f);
    up = f4(-1e32f, -1e32f, -1e32f);
    box_add(lo, up, s.x[t.x]);
    box_add(lo, up, s.x[t.y]);
    box_add(lo, up, s.x[t.z]);
    return lo;
}

ADMM_DEV float4 edge_box_lo(const DevScene& s, int o, float4& up) {
    const int2 e = s.se[o];
    float4 lo = f4(1e32f, 1e32f, 1e32f);
    up = f4(-1e32f, -1e32f, -1e32f);
    box_add(lo, up, s.x[e.x]);
    box_add(lo, up, s.x[e.y]);
    return lo;
}

// Candidate triangles of surface vertex position P (lane `sub` of the group).
template <class F>
ADMM_DEV void grid_walk_vf(const DevScene& s, float4 P, int sub, F f) {
    const GridDev& g = s.grid;
    const float gap = s.thickness;
    int3 a, b;
    grid_query_range(P, P, gap, g.inv_c, a, b);
    if (grid_range_small(a, b)) {
        const int nc = grid_cells(a, b);
        for (int ci = sub; ci < nc; ci += kQueryLanes) {
            const int3 c = grid_cell_at(a, b, ci);
            const int bk = grid_bucket(c.x, c.y, c.z, 0, g.hmask);
            const unsigned long long key = grid_cell_key(c.x, c.y, c.z);
            const int k1 = g.start[bk + 1];
            const int qfirst = (c.x == a.x ? 1 : 0) | (c.y == a.y ? 2 : 0) | (c.z == a.z ? 4 : 0);
            for (int k = g.start[bk]; k < k1; k++) {
                if (g.ent_key[k] != key) continue;  // another cell of the bucket
                const float4 up = g.ent_up[k];
                // once per pair: this cell is the first of the query's or of the element's range on every axis
                if (((qfirst | __float_as_int(up.w)) & 7) != 7) continue;
                const float4 lo = g.ent_lo[k];
                if (!box_overlap(P, P, lo, up, gap)) continue;
                f(__float_as_int(lo.w));
            }
        }
    } else {
        for (int t = sub; t < s.nst; t += kQueryLanes) {
            if (!g.mode[t]) continue;
            float4 up;
            const float4 lo = tri_box_lo(s, t, up);
            if (box_overlap(P, P, lo, up, gap)) f(t);
        }
    }
    const int nb = g.ctr[1];
    for (int j = sub; j < nb; j += kQueryLanes) {
        const int t = g.big_tri[j];
        float4 up;
        const float4 lo = tri_box_lo(s, t, up);
        if (box_overlap(P, P, lo, up, gap)) f(t);
    }
}

// Candidate partner edges of surface edge e with box [lo, up]: grid edges with a
// larger index (grid edge e), every big edge (grid edge e) or big edges with a
// larger index (big edge e).
template <class F>
ADMM_DEV void grid_walk_ee(const DevScene& s, int e, float4 lo, float4 up, int sub, F f) {
    const GridDev& g = s.grid;
    const float gap = s.thickness;
    const bool small = g.mode[s.nst + e] != 0;
    if (small) {
        int3 a, b;
        grid_query_range(lo, up, gap, g.inv_c, a, b);
        if (grid_range_small(a, b)) {
            const int nc = grid_cells(a, b);
            for (int ci = sub; ci < nc; ci += kQueryLanes) {
                const int3 c = grid_cell_at(a, b, ci);
                const int bk = grid_bucket(c.x, c.y, c.z, 1, g.hmask);
                const unsigned long long key = grid_cell_key(c.x, c.y, c.z);
                const int k1 = g.start[bk + 1];
                const int qfirst = (c.x == a.x ? 1 : 0) | (c.y == a.y ? 2 : 0) | (c.z == a.z ? 4 : 0);
                for (int k = g.start[bk]; k < k1; k++) {
                    if (g.ent_key[k] != key) continue;
                    const float4 elo = g.ent_lo[k];
                    const int o = __float_as_int(elo.w);
                    if (o <= e) continue;
                    const float4 eup = g.ent_up[k];
                    if (((qfirst | __float_as_int(eup.w)) & 7) != 7 || !box_overlap(lo, up, elo, eup, gap)) continue;
                    f(o);
                }
            }
        } else {
            for (int o = e + 1 + sub; o < s.nse; o += kQueryLanes) {
                if (!g.mode[s.nst + o]) continue;
                float4 oup;
                const float4 olo = edge_box_lo(s, o, oup);
                if (box_overlap(lo, up, olo, oup, gap)) f(o);
            }
        }
    }
    const int nb = g.ctr[2];
    for (int j = sub; j < nb; j += kQueryLanes) {
        const int o = g.big_edge[j];
        if (o == e || (!small && o < e)) continue;
        float4 oup;
        const float4 olo = edge_box_lo(s, o, oup);
        if (box_overlap(lo, up, olo, oup, gap)) f(o);  // the overlap rule is symmetric
    }
}

// ---------------------------------------------------------------------------
// Cheap distance filters in front of the exact narrow phase.  Closest points by
// the Voronoi-region construction (point-triangle) and the clamped-parameter
// construction (segment-segment), in ordinary FP32 arithmetic.  A pair is
// dropped only when this distance exceeds 1.1 x thickness plus 1e-5 of the
// largest coordinate -- orders of magnitude above the rounding of either
// computation -- so the exact predicate (d < thickness) could not have accepted
// it; non-finite intermediate values never drop a pair.  On flat cloth most
// box-overlapping non-adjacent pairs are neighbours a cell apart, and this
// keeps them out of the heavy non-contracting narrow phase.
// ---------------------------------------------------------------------------
ADMM_DEV float d3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

ADMM_DEV float fast_pt_dist2(float4 p, float4 a, float4 b, float4 c) {
    const float4 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
    const float q1 = d3(ab, ap), q2 = d3(ac, ap);
    float4 x;
    if (q1 <= 0.f && q2 <= 0.f) {
        x = a;
    } else {
        const float4 bp = sub3(p, b);
        const float q3 = d3(ab, bp), q4 = d3(ac, bp);
        const float4 cp = sub3(p, c);
        const float q5 = d3(ab, cp), q6 = d3(ac, cp);
        const float vc = q1 * q4 - q3 * q2, vb = q5 * q2 - q1 * q6, va = q3 * q6 - q5 * q4;
        if (q3 >= 0.f && q4 <= q3) {
            x = b;
        } else if (vc <= 0.f && q1 >= 0.f && q3 <= 0.f) {
            x = add3(a, scale3(ab, q1 / (q1 - q3)));
        } else if (q6 >= 0.f && q5 <= q6) {
            x = c;
        } else if (vb <= 0.f && q2 >= 0.f && q6 <= 0.f) {
            x = add3(a, scale3(ac, q2 / (q2 - q6)));
        } else if (va <= 0.f && (q4 - q3) >= 0.f && (q5 - q6) >= 0.f) {
            x = add3(b, scale3(sub3(c, b), (q4 - q3) / ((q4 - q3) + (q5 - q6))));
        } else {
            const float den = 1.f / (va + vb + vc);
            x = add3(a, add3(scale3(ab, vb * den), scale3(ac, vc * den)));
        }
    }
    const float4 d = sub3(p, x);
    return d3(d, d);
}

ADMM_DEV float fast_ee_dist2(float4 p1, float4 q1, float4 p2, float4 q2) {
    const float4 u = sub3(q1, p1), v = sub3(q2, p2), w = sub3(p1, p2);
    const float a = d3(u, u), e = d3(v, v), f = d3(v, w);
    float sp, tp;
    const float tiny = 1e-30f;
    if (a <= tiny && e <= tiny) {
        sp = tp = 0.f;
    } else if (a <= tiny) {
        sp = 0.f;
        tp = fminf(fmaxf(f / e, 0.f), 1.f);
    } else {
        const float c = d3(u, w);
        if (e <= tiny) {
            tp = 0.f;
            sp = fminf(fmaxf(-c / a, 0.f), 1.f);
        } else {
            const float b = d3(u, v), den = a * e - b * b;
            sp = den > 0.f ? fminf(fmaxf((b * f - c * e) / den, 0.f), 1.f) : 0.f;
            tp = (b * sp + f) / e;
            if (tp < 0.f) {
                tp = 0.f;
                sp = fminf(fmaxf(-c / a, 0.f), 1.f);
            } else if (tp > 1.f) {
                tp = 1.f;
                sp = fminf(fmaxf((b - c) / a, 0.f), 1.f);
            }
        }
    }
    const float4 d = sub3(add3(p1, scale3(u, sp)), add3(p2, scale3(v, tp)));
    return d3(d, d);
}

ADMM_DEV bool surely_apart(float d2, float thickness, float4 a, float4 b, float4 c, float4 d) {
    const float r = fmaxf(fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fabsf(b.x))),
                          fmaxf(fmaxf(fabsf(b.y), fabsf(b.z)), fmaxf(fmaxf(fabsf(c.x), fabsf(c.y)),
                                                                      fmaxf(fabsf(c.z), fmaxf(fmaxf(fabsf(d.x), fabsf(d.y)), fabsf(d.z))))));
    const float lim = 1.1f * thickness + 1e-5f * r;
    return d2 > lim * lim;  // false for NaN
}

// Narrow phase of vertex v against triangle f (region 0, 0 <= d < thickness).
ADMM_DEV bool grid_hit_vf(const DevScene& s, int v, float4 P, int f, int4& ids, NpResult& r) {
    const int4 tri = s.st[f];
    if (v == tri.x || v == tri.y || v == tri.z) return false;
    ids = make_int4(v, tri.x, tri.y, tri.z);
    const float4 a = s.x[tri.x], b = s.x[tri.y], c = s.x[tri.z];
    if (surely_apart(fast_pt_dist2(P, a, b, c), s.thickness, P, a, b, c)) return false;
    return narrow_pt(P, a, b, c, r) && r.dist < s.thickness && r.dist >= 0.f;
}

// Narrow phase of edges e and o (no shared vertex), lower index first.
ADMM_DEV bool grid_hit_ee(const DevScene& s, int e, int o, int4& ids, NpResult& r) {
    const int2 ed = s.se[e], od = s.se[o];
    if (ed.x == od.x || ed.x == od.y || ed.y == od.x || ed.y == od.y) return false;
    const int2 lo = o > e ? ed : od, hi = o > e ? od : ed;
    ids = make_int4(lo.x, lo.y, hi.x, hi.y);
    const float4 p0 = s.x[lo.x], p1 = s.x[lo.y], q0 = s.x[hi.x], q1 = s.x[hi.y];
    if (surely_apart(fast_ee_dist2(p0, p1, q0, q1), s.thickness, p0, p1, q0, q1)) return false;
    return narrow_ee(p0, p1, q0, q1, r) && r.dist < s.thickness && r.dist >= 0.f;
}

// Count (WRITE = false: qcount) or write (WRITE = true: at qoff, then sorted by
// partner) the pairs of every query: surface vertices first, then edges.
template <bool WRITE>
__global__ void __launch_bounds__(128) k_grid_query(DevScene s) {
    ADMM_PDL_PROLOGUE();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = t / kQueryLanes, sub = t % kQueryLanes;
    if (q >= s.nsv + s.nse) return;  // whole groups leave together
    const unsigned gmask = 0xffu << (threadIdx.x & 31 & ~(kQueryLanes - 1));
    const bool vf = q < s.nsv;
    const int e = q - s.nsv;
    int v = 0;
    float4 P = f4(0.f, 0.f, 0.f), lo = P, up = P;
    if (vf) {
        v = s.sv[q];
        P = s.x[v];
    } else {
        lo = edge_box_lo(s, e, up);
    }
    // Count pass: walk the grid, record up to kQueryHits partners per lane in
    // qhits and the lane's hit count in qlane.  Write pass: take the recorded
    // partners (the walk again only for a lane with more hits).
    int* my_hits = s.grid.qhits + (size_t)t * kQueryHits;
    int n = 0;
    if (!WRITE) {
        auto consider = [&](int partner) {
            int4 ids;
            NpResult r;
            if (vf ? grid_hit_vf(s, v, P, partner, ids, r) : grid_hit_ee(s, e, partner, ids, r)) {
                if (n < kQueryHits) my_hits[n] = partner;
                n++;
            }
        };
        if (vf) grid_walk_vf(s, P, sub, consider);
        else grid_walk_ee(s, e, lo, up, sub, consider);
        s.grid.qlane[t] = n;
    } else {
        n = s.grid.qlane[t];
    }
    // group sum / exclusive prefix of the lane counts
    int incl = n;
#pragma unroll
    for (int o = 1; o < kQueryLanes; o <<= 1) {
        const int y = __shfl_up_sync(gmask, incl, o, kQueryLanes);
        if (sub >= o) incl += y;
    }
    const int total = __shfl_sync(gmask, incl, kQueryLanes - 1, kQueryLanes);
    if (!WRITE) {
        if (sub == 0) s.qcount[q] = total;
        return;
    }
    const int base = s.qoff[q];
    int slot = base + incl - n;
    auto emit = [&](int partner) {
        int4 ids;
        NpResult r;
        const bool hit = vf ? grid_hit_vf(s, v, P, partner, ids, r) : grid_hit_ee(s, e, partner, ids, r);
        if (hit) {
            if (slot < s.cap) {
                write_contact(s, slot, ids, r, !vf);
                s.grid.qkey[slot] = partner;
            }
            slot++;
        }
    };
    if (n <= kQueryHits) {
        for (int k = 0; k < n; k++) emit(my_hits[k]);
    } else if (vf) {
        grid_walk_vf(s, P, sub, emit);
    } else {
        grid_walk_ee(s, e, lo, up, sub, emit);
    }
    __syncwarp(gmask);
    if (sub == 0) {
        const int end = min(base + total, s.cap);
        if (end - base > 1) grid_sort_segment(s, base, end);
    }
}

}  // namespace admm
