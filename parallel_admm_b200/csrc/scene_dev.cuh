// scene_dev.cuh -- device-side view of one ADMM scene (all pointers device).
#pragma once
#include "common.cuh"

namespace admm {

constexpr int kStackDepth = 64;     // BVH traversal stack (lbvh.cu:1698 uses 64)

// Sliced ELL with `lanes` (T) threads per row: slices of 32/T rows, one warp per
// slice; entry k of local row lr at ptr[s] + (k/T)*32 + (k%T)*(32/T) + lr.  Slot
// lr of slice s holds row rowid[s*32/T + lr] (rows reordered by length within
// windows of 32), or row s*32/T + lr without rowid.
struct SlicedEll {
    int rows = 0;
    int nslices = 0;
    int lanes = 1;
    const int* ptr = nullptr;    // [nslices+1] offsets (multiples of kSlice)
    const int* col = nullptr;
    const float* val = nullptr;
    const int* rowid = nullptr;  // [nslices * 32/T] row of each slot (null: slot = row)
};

struct BvhDev {
    int n = 0;                   // leaves
    float4* box_lo = nullptr;    // [2n-1]: internal nodes [0, n-1), leaves [n-1, 2n-1)
    float4* box_up = nullptr;
    int* left = nullptr;         // [n-1]
    int* right = nullptr;        // [n-1]
    int* parent = nullptr;       // [2n-1]
    int* leaf_elem = nullptr;    // [n] element id of sorted leaf i
    uint32_t* flags = nullptr;   // [n-1] refit arrival counters
    unsigned long long* keys = nullptr;   // [n] sort keys
    unsigned long long* keys_alt = nullptr;
    int* vals = nullptr;         // [n] element ids (sort payload)
    int* vals_alt = nullptr;
    float4* elem_lo = nullptr;   // [n] unsorted element boxes
    float4* elem_up = nullptr;
    uint32_t* scene = nullptr;   // [6] ordered-float min xyz, max xyz
    // Internal node i as one 64-byte record: node4[4i+0] = left child box lower
    // (w = left index), [4i+1] = left upper, [4i+2] = right lower (w = right
    // index), [4i+3] = right upper.  One load per traversal level.
    float4* node4 = nullptr;     // [4(n-1)]
};

// Row tiles of the two-sweep Jacobi kernel (see build_tiles in setup.hpp).
struct TileSet {
    int ntiles = 0;
    const int *row0 = nullptr, *nlocal = nullptr, *nown = nullptr;
    const int *s1_0 = nullptr, *s1_n = nullptr, *s2_0 = nullptr, *s2_n = nullptr;
    const int* trow = nullptr;   // local row -> global row (-1 = padding)
    SlicedEll e1, e2;            // phase 1 (global columns), phase 2 (tile-local columns)
};

// Work split and dependency lists of the persistent global-step kernel.
struct PersistPlan {
    int blocks = 0;                // one per SM at most (cooperative launch)
    int rows_per_block = 0;        // multiple of 32
    const int* dep_ptr = nullptr;  // [blocks + 1]
    const int* dep_idx = nullptr;  // blocks whose rows share a matrix entry with this block's rows
    unsigned* epoch = nullptr;     // [blocks] sweeps completed (monotone, wraps)
    int spin_limit = 0;            // polls before a wait gives up
};

// Uniform-grid broad phase: hash table of (cell, element type) buckets.
struct GridDev {
    float inv_c = 0.f;             // 1 / cell edge
    int hmask = 0;                 // buckets - 1 (power of two)
    int cap = 0;                   // entry capacity
    int* cnt = nullptr;            // [buckets] entries per bucket (zero between DCDs)
    int* start = nullptr;          // [buckets + 1] bucket offsets
    float4* ent_lo = nullptr;      // [cap] element box lo, w = element index (int bits)
    float4* ent_up = nullptr;      // [cap] element box up, w = first-cell bits (x 1, y 2, z 4)
    unsigned long long* ent_key = nullptr;  // [cap] key of the cell the entry was made for
    int* ctr = nullptr;            // [4] entries reserved, big triangles, big edges
    int* big_tri = nullptr;        // [n surface triangles]
    int* big_edge = nullptr;       // [n surface edges]
    int* mode = nullptr;           // [triangles + edges] 1 = in the grid, 0 = big list
    int* qkey = nullptr;           // [contact capacity] partner index per contact slot
    int* qhits = nullptr;          // [queries * kQueryHitsMax] partners found by the count pass
};

struct DevScene {
    int n = 0, nd = 0, m = 0;
    int ntri = 0, ntet = 0, nbend = 0, npin = 0;
    int tri_sr = 0, tet_sr = 0, bend_sr = 0, pin_sr = 0;
    float dt = 0, dt_inv = 0, g = 0, mu = 0, eps = 0, gam = 0, thickness = 0;
    int contact = 0;
    int cpu_contact = 0;  // contact predicates of the CPU backend (ProximalQuery)
    int cpu_backend = 0;  // solver semantics of the CPU backend (damping, S_c, serial Gauss-Seidel)
    // CPU backend's damping matrix (off-diagonal CSR + diagonal) for b_ini = Damp x0
    const int* dmp_start = nullptr;
    const int* dmp_col = nullptr;
    const float* dmp_val = nullptr;
    const float* dmp_diag = nullptr;
    // vertex state (float4 rows, w unused)
    float4 *x = nullptr, *x0 = nullptr, *v = nullptr, *p = nullptr, *mxt = nullptr;
    float4 *b = nullptr, *uc = nullptr, *xprev = nullptr, *jac[2] = {nullptr, nullptr};
    const float* mass = nullptr;
    const int* fixed = nullptr;
    const float* dt2wc = nullptr;    // [nd] h^2 w_c (0 off the contact surface)
    const float* cw = nullptr;       // [n] w_c
    const float* cwinv = nullptr;    // [n] 1/w_c (0 for static vertices)
    // constraints
    const int4* tri_inds = nullptr;
    const float4* tri_binv = nullptr;     // (B00, B01, B10, B11)
    const int4* tet_inds = nullptr;
    const float4* tet_b0 = nullptr;       // Binv rows (xyz)
    const float4* tet_b1 = nullptr;
    const float4* tet_b2 = nullptr;
    const int* bend_off = nullptr;
    const int* bend_inds = nullptr;
    const float* bend_coef = nullptr;
    const float* bend_rest = nullptr;
    const int* pin_inds = nullptr;
    const float4* pin_pos = nullptr;
    const float* wrow = nullptr;          // [m] w per row
    float4 *z = nullptr, *ue = nullptr, *y = nullptr;   // y = z - Ue
    // matrices
    SlicedEll A;                          // off-diagonal part of the system matrix
    const float* a_diag = nullptr;
    SlicedEll R;                          // h^2 D^T W^2 (rows = dynamic vertices)
    // contacts
    int cap = 0;
    int* nc = nullptr;                    // [1] device contact count (clamped to cap)
    int* nc_raw = nullptr;                // [1] unclamped count
    int* err = nullptr;                   // [4] error flags: overflow, stack, nan, wait timeout
    int4* pairs = nullptr;
    float4* bary = nullptr;
    float4* nrm = nullptr;                // normal xyz, w = h_cN - thickness
    float4* point = nullptr;
    float4* gamma = nullptr;              // Gamma_c per contact slot
    float4* kc = nullptr;
    float4* rc = nullptr;
    float* cmu = nullptr;                 // [cap] friction coefficient per contact
    const float* vmu = nullptr;           // [n] per-vertex coefficient, or null
    float4* du = nullptr;
    float4* du2 = nullptr;  // [cap] second buffer of the fused projection passes
    float4* p2 = nullptr;   // [n] second buffer of p in the fused projection passes
    int* vcnt = nullptr;                  // [n] contacts per vertex
    int* vfill = nullptr;                 // [n]
    int* vstart = nullptr;                // [n+1]
    int* vlist = nullptr;                 // [4*cap] contact*4 + slot, sorted per vertex
    float2* ginc = nullptr;               // [4*cap] (contact as int bits, Gamma_c,i) in list order
    int* vtmp = nullptr;                  // [4*cap] incidence lists before sorting
    int* tpos = nullptr;                  // [n] position of a vertex in the touched list
    int* tv = nullptr;                    // [n] vertices with contacts, ascending
    int* ntv = nullptr;                   // [1] their number
    int4* cinc = nullptr;                 // [4*cap] per contact corner: (vertex, list begin, list end, 0)
    int4* tvr = nullptr;                  // [n] per touched vertex, in tv order: (vertex, list begin, list end, 0)
    // collision geometry
    int nst = 0, nse = 0, nsv = 0;
    const int4* st = nullptr;             // surface triangles (w unused)
    const int2* se = nullptr;             // surface edges
    const int* sv = nullptr;              // surface vertices
    BvhDev bf, be;                        // face tree, edge tree
    GridDev grid;                         // uniform-grid broad phase
    int* qcount = nullptr;                // [nsv + nse] per-query pair counts
    int* qoff = nullptr;                  // [nsv + nse + 1] exclusive offsets
    int* scan_tmp = nullptr;              // block sums for scans
    // residuals: [0] primal^2, [1] dual^2, [2] scale^2
    double* res = nullptr;
    double* res_part = nullptr;           // [3 x residual blocks] per-block partial sums
    int* done = nullptr;
};

}  // namespace admm
