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
// Queries: G consecutive lanes of a warp serve one query (G = 8, 16 or 32).
// The entries of all cells of the query's range are numbered consecutively (an
// inclusive scan of the bucket sizes over the group, G cells at a time) and
// lane k of the group takes entries k, k + G, ..., so every lane has the same
// share whatever the cell sizes; an entry's cell key, box and first-cell bits
// are loaded together.  Candidates that pass the cell-key, once-per-pair and
// box tests are queued in shared memory and handed to the narrow phase G at a
// time, so that it runs on full groups.  G = 32 suits a few thousand queries
// (latency bound: more lanes per query shorten each query's chain of loads);
// G = 8 suits millions (throughput bound: less scan and queue work per entry).
// ---------------------------------------------------------------------------
constexpr int kQueryThreads = 128;  // block size of the query kernels
constexpr int kQueryHitsMax = 32;   // partners the count pass records per query

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

// The lanes of one query: sub = lane within the group, mask = the group's lanes.
template <int G>
struct QueryGroup {
    int sub;
    unsigned mask;
    ADMM_DEV QueryGroup() {
        const int lane = threadIdx.x & 31;
        sub = lane % G;
        mask = G == 32 ? ~0u : (((1u << G) - 1u) << (lane - sub));
    }
    // bits of the group's lanes with pred set, lane `sub` of the group at bit `sub`
    ADMM_DEV unsigned ballot(bool pred) const {
        const unsigned m = __ballot_sync(mask, pred);
        return G == 32 ? m : (m >> ((threadIdx.x & 31) - sub)) & ((1u << G) - 1u);
    }
    ADMM_DEV unsigned below() const { return (1u << sub) - 1u; }
};

// Candidate partners of one group waiting for the narrow phase (2G slots in
// shared memory; the fill n is the same in every lane of the group).
struct GridQueue {
    int* buf;
    int n;
};

// Queues the partner of every lane with ok set (called by the whole group);
// once G or more wait, hands the first G to narrow(partner, true).
template <int G, class F>
ADMM_DEV void grid_queue_push(const QueryGroup<G>& grp, GridQueue& q, bool ok, int partner, F& narrow) {
    const unsigned m = grp.ballot(ok);
    if (ok) q.buf[q.n + __popc(m & grp.below())] = partner;
    q.n += __popc(m);
    if (q.n >= G) {
        __syncwarp(grp.mask);
        const int p = q.buf[grp.sub];
        if (grp.sub < q.n - G) q.buf[grp.sub] = q.buf[G + grp.sub];
        __syncwarp(grp.mask);
        q.n -= G;
        narrow(p, true);
    }
}

template <int G, class F>
ADMM_DEV void grid_queue_drain(const QueryGroup<G>& grp, GridQueue& q, F& narrow) {
    if (q.n == 0) return;
    __syncwarp(grp.mask);
    const bool valid = grp.sub < q.n;
    const int p = valid ? q.buf[grp.sub] : 0;
    __syncwarp(grp.mask);
    q.n = 0;
    narrow(p, valid);
}

// The group's walk of one query.  Vertex query (vf): position P = lo = up
// against the triangles.  Edge query: edge e with box [lo, up] against grid
// edges with a larger index (grid edge e), every big edge (grid edge e) or big
// edges with a larger index (big edge e).  Grid part: the cells of the query's
// range, or every grid element of the type when the range is too large.
template <int G, class F>
ADMM_DEV void grid_walk(const DevScene& s, const QueryGroup<G>& grp, bool vf, int e, float4 lo, float4 up,
                        GridQueue& q, F& narrow) {
    const GridDev& g = s.grid;
    const float gap = s.thickness;
    const int sub = grp.sub;
    const unsigned gm = grp.mask;
    const int type = vf ? 0 : 1;
    const bool small = vf || g.mode[s.nst + e] != 0;
    if (small) {
        int3 a, b;
        grid_query_range(lo, up, gap, g.inv_c, a, b);
        if (grid_range_small(a, b)) {
            const int nc = grid_cells(a, b);
            for (int c0 = 0; c0 < nc; c0 += G) {
                int cnt = 0, d = 0, qfirst = 0;
                unsigned long long key = 0ull;
                if (c0 + sub < nc) {
                    const int3 c = grid_cell_at(a, b, c0 + sub);
                    const int bk = grid_bucket(c.x, c.y, c.z, type, g.hmask);
                    d = g.start[bk];
                    cnt = g.start[bk + 1] - d;
                    key = grid_cell_key(c.x, c.y, c.z);
                    qfirst = (c.x == a.x ? 1 : 0) | (c.y == a.y ? 2 : 0) | (c.z == a.z ? 4 : 0);
                }
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < G; o <<= 1) {
                    const int y = __shfl_up_sync(gm, incl, o, G);
                    if (sub >= o) incl += y;
                }
                d -= incl - cnt;  // entry number k of the round lies at d of its cell + k
                const int tot = __shfl_sync(gm, incl, G - 1, G);
                for (int k0 = 0; k0 < tot; k0 += G) {
                    const int k = k0 + sub;
                    // the cell of entry k: the first lane of the group whose inclusive count exceeds k
                    int j = 0;
#pragma unroll
                    for (int st = G / 2; st >= 1; st >>= 1) {
                        if (__shfl_sync(gm, incl, j + st - 1, G) <= k) j += st;
                    }
                    const int dj = __shfl_sync(gm, d, j, G);
                    const int fj = __shfl_sync(gm, qfirst, j, G);
                    const unsigned long long kj = __shfl_sync(gm, key, j, G);
                    bool ok = false;
                    int partner = 0;
                    if (k < tot) {
                        const int ent = dj + k;
                        const unsigned long long ek = g.ent_key[ent];
                        const float4 eup = g.ent_up[ent];
                        const float4 elo = g.ent_lo[ent];
                        partner = __float_as_int(elo.w);
                        // same cell (not another of the bucket); larger edge index; once per pair:
                        // this cell is the first of the query's or of the element's range on every axis
                        ok = ek == kj && (vf || partner > e) && ((fj | __float_as_int(eup.w)) & 7) == 7 &&
                             (s.cpu_contact || box_overlap(lo, up, elo, eup, gap));
                    }
                    grid_queue_push(grp, q, ok, partner, narrow);
                }
            }
        } else {
            const int n = vf ? s.nst : s.nse;
            for (int t0 = vf ? 0 : e + 1; t0 < n; t0 += G) {
                const int t = t0 + sub;
                bool ok = false;
                if (t < n && g.mode[vf ? t : s.nst + t]) {
                    float4 eup;
                    const float4 elo = vf ? tri_box_lo(s, t, eup) : edge_box_lo(s, t, eup);
                    ok = s.cpu_contact || box_overlap(lo, up, elo, eup, gap);
                }
                grid_queue_push(grp, q, ok, t, narrow);
            }
        }
    }
    const int nb = g.ctr[1 + type];
    for (int j0 = 0; j0 < nb; j0 += G) {
        const int j = j0 + sub;
        bool ok = false;
        int o = 0;
        if (j < nb) {
            o = vf ? g.big_tri[j] : g.big_edge[j];
            if (vf || (o != e && (small || o > e))) {
                float4 oup;
                const float4 olo = vf ? tri_box_lo(s, o, oup) : edge_box_lo(s, o, oup);
                ok = s.cpu_contact || box_overlap(lo, up, olo, oup, gap);  // the overlap rule is symmetric
            }
        }
        grid_queue_push(grp, q, ok, o, narrow);
    }
    grid_queue_drain(grp, q, narrow);
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
// Narrow phase of vertex v against triangle f: the GPU backend's (region 0,
// 0 <= d < thickness) or, with cpu_contact, the CPU backend's (no pair of two
// static elements, any closest point, d <= thickness).
ADMM_DEV bool grid_hit_vf(const DevScene& s, int v, float4 P, int f, int4& ids, NpResult& r) {
    const int4 tri = s.st[f];
    if (v == tri.x || v == tri.y || v == tri.z) return false;
    if (s.cpu_contact && v >= s.nd && tri.x >= s.nd) return false;
    ids = make_int4(v, tri.x, tri.y, tri.z);
    const float4 a = s.x[tri.x], b = s.x[tri.y], c = s.x[tri.z];
    if (surely_apart(fast_pt_dist2(P, a, b, c), s.thickness, P, a, b, c)) return false;
    if (s.cpu_contact) {
        closest_pt_all(P, a, b, c, r);
        return r.dist <= s.thickness;
    }
    return narrow_pt(P, a, b, c, r) && r.dist < s.thickness && r.dist >= 0.f;
}

// Narrow phase of edges e and o (no shared vertex), lower index first.
// Narrow phase of edges e and o (no shared vertex), lower index first: the GPU
// backend's (region 0) or, with cpu_contact, the CPU backend's (no pair of two
// static edges, d < thickness unless both closest points are end points).
ADMM_DEV bool grid_hit_ee(const DevScene& s, int e, int o, int4& ids, NpResult& r) {
    const int2 ed = s.se[e], od = s.se[o];
    if (ed.x == od.x || ed.x == od.y || ed.y == od.x || ed.y == od.y) return false;
    const int2 lo = o > e ? ed : od, hi = o > e ? od : ed;
    if (s.cpu_contact && lo.x >= s.nd && hi.x >= s.nd) return false;
    ids = make_int4(lo.x, lo.y, hi.x, hi.y);
    const float4 p0 = s.x[lo.x], p1 = s.x[lo.y], q0 = s.x[hi.x], q1 = s.x[hi.y];
    if (surely_apart(fast_ee_dist2(p0, p1, q0, q1), s.thickness, p0, p1, q0, q1)) return false;
    if (s.cpu_contact) {
        closest_ee_all(p0, p1, q0, q1, r);
        const bool corner = (r.bary[0] == 0.f || r.bary[0] == 1.f) && (r.bary[1] == 0.f || r.bary[1] == 1.f);
        return r.dist < s.thickness && !corner;
    }
    return narrow_ee(p0, p1, q0, q1, r) && r.dist < s.thickness && r.dist >= 0.f;
}

// Count (WRITE = false) or write (WRITE = true) the pairs of every query, G
// lanes per query: surface vertices first, then edges.  The count pass stores
// the query's pair count in qcount and up to kQueryHitsMax partners in qhits.
// The write pass places each recorded partner at qoff + its rank among the
// query's partners, so the segment comes out sorted by partner; a query with
// more partners than were recorded walks the grid again, writes in walk order
// and sorts its segment.
template <bool WRITE, int G>
ADMM_DEV void grid_query(DevScene& s) {
    ADMM_PDL_PROLOGUE();
    __shared__ int qbuf[kQueryThreads * 2];
    const QueryGroup<G> grp;
    const int q = (blockIdx.x * kQueryThreads + threadIdx.x) / G;
    if (q >= s.nsv + s.nse) return;  // whole groups leave together
    const bool vf = q < s.nsv;
    const int e = q - s.nsv;
    int v = 0;
    float4 lo, up;
    if (vf) {
        v = s.sv[q];
        lo = up = s.x[v];
    } else {
        lo = edge_box_lo(s, e, up);
    }
    GridQueue gq{qbuf + 2 * (threadIdx.x - grp.sub), 0};
    int* qh = s.grid.qhits + (size_t)q * kQueryHitsMax;
    int nhit = 0;  // the same in every lane of the group
    if (!WRITE) {
        auto narrow = [&](int partner, bool valid) {
            int4 ids;
            NpResult r;
            const bool hit = valid && (vf ? grid_hit_vf(s, v, lo, partner, ids, r) : grid_hit_ee(s, e, partner, ids, r));
            const unsigned m = grp.ballot(hit);
            const int k = nhit + __popc(m & grp.below());
            if (hit && k < kQueryHitsMax) qh[k] = partner;
            nhit += __popc(m);
        };
        grid_walk(s, grp, vf, e, lo, up, gq, narrow);
        if (grp.sub == 0) s.qcount[q] = nhit;
        return;
    }
    const int total = s.qcount[q];
    if (total == 0) return;
    const int base = s.qoff[q];
    if (total <= kQueryHitsMax) {
        for (int k = grp.sub; k < total; k += G) {
            const int partner = qh[k];
            int rank = 0;
            for (int j = 0; j < total; j++) rank += qh[j] < partner ? 1 : 0;
            int4 ids;
            NpResult r;
            const bool hit = vf ? grid_hit_vf(s, v, lo, partner, ids, r) : grid_hit_ee(s, e, partner, ids, r);
            const int slot = base + rank;
            if (hit && slot < s.cap) write_contact(s, slot, ids, r, !vf);
        }
        return;
    }
    auto emit = [&](int partner, bool valid) {
        int4 ids;
        NpResult r;
        const bool hit = valid && (vf ? grid_hit_vf(s, v, lo, partner, ids, r) : grid_hit_ee(s, e, partner, ids, r));
        const unsigned m = grp.ballot(hit);
        const int slot = base + nhit + __popc(m & grp.below());
        if (hit && slot < s.cap) {
            write_contact(s, slot, ids, r, !vf);
            s.grid.qkey[slot] = partner;
        }
        nhit += __popc(m);
    };
    grid_walk(s, grp, vf, e, lo, up, gq, emit);
    __syncwarp(grp.mask);
    if (grp.sub == 0) {
        const int end = min(base + total, s.cap);
        if (end - base > 1) grid_sort_segment(s, base, end);
    }
}

template <bool WRITE, int G>
__global__ void __launch_bounds__(kQueryThreads) k_grid_query(DevScene s) {
    grid_query<WRITE, G>(s);
}

// The count pass of a throughput-bound detection (G = 8), capped at 48
// registers (10 blocks per SM): more resident warps hide its load latency
// better than the few spilled registers cost (4.2 M queries of the 4 x 512^2
// sheets: 46.6 against 52.6 ms of DCD per substep).  The other passes keep the
// compiler's register choice.
__global__ void __launch_bounds__(kQueryThreads, 10) k_grid_count8(DevScene s) {
    grid_query<false, 8>(s);
}

}  // namespace admm
