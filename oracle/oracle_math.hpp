// oracle_math.hpp -- TEST INFRASTRUCTURE ONLY (the oracle).  Not part of the
// product: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// may load the oracle, and only as the checker.
//
// Small-vector math, the 3x3 SVD and the narrow-phase predicates of the
// reference, restated on the CPU.  Built with -ffp-contract=off so every float
// operation is one IEEE round-to-nearest operation, in the order written.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>

namespace orc {

template <class R> struct V3 {
    R x, y, z;
};
template <class R> inline V3<R> mk(R a, R b, R c) { return V3<R>{a, b, c}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
// dot in Eigen's fixed-size unrolled order ((x*x + y*y) + z*z)
template <class R> inline R dot(V3<R> a, V3<R> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R norm(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V3<R> normalized(V3<R> a) {
    R n2 = dot(a, a);
    if (n2 > R(0)) { R n = std::sqrt(n2); return {a.x / n, a.y / n, a.z / n}; }
    return a;
}

// ---------------------------------------------------------------------------
// Narrow phase: src/mutils/dist_g.cuh:29-252 (dcdPT) and 257-513 (dcdEE).
// Only region 0 (interior closest points) is accepted by the reference GPU
// path; every other region returns distance = -10.  The arithmetic below is
// the reference's operation sequence for the accepted region and for every
// branch decision that leads to it.
// ---------------------------------------------------------------------------
template <class R> struct Result {
    R distance, sqrDistance;
    R bary[3];
    V3<R> closest[2];
};

template <class R>
inline Result<R> dcd_pt(V3<R> point, V3<R> t0, V3<R> t1, V3<R> t2) {
    Result<R> res{};
    const R zero = 0;
    V3<R> diff = t0 - point;
    V3<R> edge0 = t1 - t0;
    V3<R> edge1 = t2 - t0;
    R a00 = dot(edge0, edge0);
    R a01 = dot(edge0, edge1);
    R a11 = dot(edge1, edge1);
    R b0 = dot(diff, edge0);
    R b1 = dot(diff, edge1);
    R det = std::max(a00 * a11 - a01 * a01, zero);
    R s = a01 * b1 - a11 * b0;
    R t = a01 * b0 - a00 * b1;
    // region 0 <=> (s + t <= det) && !(s < 0) && !(t < 0)
    if (!(s + t <= det) || s < zero || t < zero) {
        res.distance = R(-10);
        return res;
    }
    s /= det;
    t /= det;
    res.closest[0] = point;
    res.closest[1] = (t0 + s * edge0) + t * edge1;
    diff = res.closest[0] - res.closest[1];
    res.sqrDistance = dot(diff, diff);
    res.distance = std::sqrt(res.sqrDistance);
    res.bary[0] = (R(1) - s) - t;
    res.bary[1] = s;
    res.bary[2] = t;
    return res;
}

template <class R>
inline Result<R> dcd_ee(V3<R> P0, V3<R> P1, V3<R> Q0, V3<R> Q1) {
    Result<R> res{};
    const R zero = 0;
    V3<R> P1mP0 = P1 - P0;
    V3<R> Q1mQ0 = Q1 - Q0;
    V3<R> P0mQ0 = P0 - Q0;
    R a = dot(P1mP0, P1mP0);
    R b = dot(P1mP0, Q1mQ0);
    R c = dot(Q1mQ0, Q1mQ0);
    R d = dot(P1mP0, P0mQ0);
    R e = dot(Q1mQ0, P0mQ0);
    R det = a * c - b * b;
    bool valid = false;
    R s = 0, t = 0;
    if (det > zero) {
        R bte = b * e;
        R ctd = c * d;
        if (!(bte <= ctd)) {
            s = bte - ctd;
            if (!(s >= det)) {
                R ate = a * e;
                R btd = b * d;
                if (!(ate <= btd)) {
                    t = ate - btd;
                    if (!(t >= det)) {
                        s /= det;
                        t /= det;
                        valid = true;
                    }
                }
            }
        }
    }
    if (!valid) {
        res.distance = R(-10);
        return res;
    }
    res.bary[0] = s;
    res.bary[1] = t;
    res.bary[2] = R(-10);
    res.closest[0] = P0 + s * P1mP0;
    res.closest[1] = Q0 + t * Q1mQ0;
    V3<R> diff = res.closest[0] - res.closest[1];
    res.sqrDistance = dot(diff, diff);
    res.distance = std::sqrt(res.sqrDistance);
    return res;
}

// ---------------------------------------------------------------------------
// Narrow phase of the reference's CPU backend (ProximalQuery::narrow_PT /
// narrow_EE, src/contact/narrow_phase.cpp:376-469), which calls the closest-
// point queries of David Eberly's Geometric Tools (src/mutils/distPT.h,
// distEE.h; published in "Distance Between Point and Triangle in 3D" and
// "Distance Between Two Line Segments in 3D", geometrictools.com).  Every
// region is accepted.  Point-triangle: minimise |t0 + s e0 + t e1 - p|^2 over
// the triangle by the sign of the unconstrained minimiser (s, t) and of
// s + t - det; the closest point is t0 + s e0 + t e1, barycentric
// (1 - s - t, s, t).  Segment-segment: minimise over [0,1]^2 by the signs of
// b e - c d and a e - b d (or, for parallel segments, along the edges of the
// square); parameters (s, t) are returned in bary[0..1] and bary[2] = -2 marks
// an edge-edge result, as the GPU path's results do.  The operation order is
// the reference's, so the accepted pair sets agree bit for bit.
// ---------------------------------------------------------------------------
template <class R>
inline Result<R> gt_point_triangle(V3<R> point, V3<R> t0, V3<R> t1, V3<R> t2) {
    const R zero = 0, one = 1, two = 2;
    V3<R> diff = t0 - point, e0 = t1 - t0, e1 = t2 - t0;
    const R a00 = dot(e0, e0), a01 = dot(e0, e1), a11 = dot(e1, e1);
    const R b0 = dot(diff, e0), b1 = dot(diff, e1);
    const R det = std::max(a00 * a11 - a01 * a01, zero);
    R s = a01 * b1 - a11 * b0;
    R t = a01 * b0 - a00 * b1;
    // the minimiser clamped to an edge s = 0 / t = 0 from the sign of b
    auto edge_t = [&](R& u) { u = b1 >= zero ? zero : (-b1 >= a11 ? one : -b1 / a11); };
    auto edge_s = [&](R& u) { u = b0 >= zero ? zero : (-b0 >= a00 ? one : -b0 / a00); };
    if (s + t <= det) {
        if (s < zero) {
            if (t < zero) {          // below both edges: vertex t0 region
                if (b0 < zero) {
                    t = zero;
                    s = -b0 >= a00 ? one : -b0 / a00;
                } else {
                    s = zero;
                    edge_t(t);
                }
            } else {                 // beyond edge s = 0
                s = zero;
                edge_t(t);
            }
        } else if (t < zero) {       // beyond edge t = 0
            t = zero;
            edge_s(s);
        } else {                     // interior
            s /= det;
            t /= det;
        }
    } else {
        if (s < zero) {              // beyond vertex t2
            const R q0 = a01 + b0, q1 = a11 + b1;
            if (q1 > q0) {
                const R num = q1 - q0, den = a00 - two * a01 + a11;
                if (num >= den) { s = one; t = zero; }
                else { s = num / den; t = one - s; }
            } else {
                s = zero;
                t = q1 <= zero ? one : (b1 >= zero ? zero : -b1 / a11);
            }
        } else if (t < zero) {       // beyond vertex t1
            const R q0 = a01 + b1, q1 = a00 + b0;
            if (q1 > q0) {
                const R num = q1 - q0, den = a00 - two * a01 + a11;
                if (num >= den) { t = one; s = zero; }
                else { t = num / den; s = one - t; }
            } else {
                t = zero;
                s = q1 <= zero ? one : (b0 >= zero ? zero : -b0 / a00);
            }
        } else {                     // beyond edge s + t = 1
            const R num = a11 + b1 - a01 - b0;
            if (num <= zero) { s = zero; t = one; }
            else {
                const R den = a00 - two * a01 + a11;
                if (num >= den) { s = one; t = zero; }
                else { s = num / den; t = one - s; }
            }
        }
    }
    Result<R> r{};
    r.closest[0] = point;
    r.closest[1] = (t0 + s * e0) + t * e1;
    diff = r.closest[0] - r.closest[1];
    r.sqrDistance = dot(diff, diff);
    r.distance = std::sqrt(r.sqrDistance);
    r.bary[0] = (one - s) - t;
    r.bary[1] = s;
    r.bary[2] = t;
    return r;
}

template <class R>
inline Result<R> gt_segment_segment(V3<R> P0, V3<R> P1, V3<R> Q0, V3<R> Q1) {
    const R zero = 0, one = 1;
    const V3<R> u = P1 - P0, v = Q1 - Q0, w = P0 - Q0;
    const R a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w), e = dot(v, w);
    const R det = a * c - b * b;
    R s = zero, t = zero;
    // s on [0, 1] for a fixed t edge: numerator n over a, clamped
    auto clamp_s = [&](R n) { return n <= zero ? zero : (n >= a ? one : n / a); };
    if (det > zero) {
        const R bte = b * e, ctd = c * d;
        if (bte <= ctd) {            // s <= 0
            s = zero;
            if (e <= zero) {
                t = zero;
                const R nd = -d;
                if (nd >= a) s = one;
                else if (nd > zero) s = nd / a;
            } else if (e < c) {
                t = e / c;
            } else {
                t = one;
                const R bmd = b - d;
                if (bmd >= a) s = one;
                else if (bmd > zero) s = bmd / a;
            }
        } else {
            s = bte - ctd;
            if (s >= det) {          // s >= 1
                s = one;
                const R bpe = b + e;
                if (bpe <= zero) {
                    t = zero;
                    const R nd = -d;
                    if (nd <= zero) s = zero;
                    else if (nd < a) s = nd / a;
                } else if (bpe < c) {
                    t = bpe / c;
                } else {
                    t = one;
                    const R bmd = b - d;
                    if (bmd <= zero) s = zero;
                    else if (bmd < a) s = bmd / a;
                }
            } else {                 // 0 < s < 1
                const R ate = a * e, btd = b * d;
                if (ate <= btd) {
                    t = zero;
                    s = clamp_s(-d);
                } else {
                    t = ate - btd;
                    if (t >= det) {
                        t = one;
                        s = clamp_s(b - d);
                    } else {
                        s /= det;
                        t /= det;
                    }
                }
            }
        }
    } else {                         // parallel segments
        if (e <= zero) {
            t = zero;
            s = clamp_s(-d);
        } else if (e >= c) {
            t = one;
            s = clamp_s(b - d);
        } else {
            s = zero;
            t = e / c;
        }
    }
    Result<R> r{};
    r.bary[0] = s;
    r.bary[1] = t;
    r.bary[2] = R(-2);
    r.closest[0] = P0 + s * u;
    r.closest[1] = Q0 + t * v;
    const V3<R> diff = r.closest[0] - r.closest[1];
    r.sqrDistance = dot(diff, diff);
    r.distance = std::sqrt(r.sqrDistance);
    return r;
}

// AABB overlap with gap (lbvh.cu:43-49)
template <class R> struct Box {
    V3<R> lo, up;
};
template <class R> inline bool overlap(const Box<R>& l, const Box<R>& r, R gap) {
    if ((r.lo.x - l.up.x) >= gap || (l.lo.x - r.up.x) >= gap) return false;
    if ((r.lo.y - l.up.y) >= gap || (l.lo.y - r.up.y) >= gap) return false;
    if ((r.lo.z - l.up.z) >= gap || (l.lo.z - r.up.z) >= gap) return false;
    return true;
}

// ---------------------------------------------------------------------------
// 3x3 SVD with the sign convention of McAdams et al., "Computing the Singular
// Value Decomposition of 3x3 matrices with minimal branching and elementary
// floating point operations", UW-Madison TR1690 (2011): U and V are proper
// rotations, sigma1 >= sigma2 >= |sigma3|, only sigma3 may be negative.
// This is the convention of the reference's svd (src/mutils/svd_fast3.cuh:37).
// Method (not the TR's approximate rotations): cyclic Jacobi on F^T F with
// exact rotations (Golub & Van Loan, Alg. 8.5.2) -> V, sort, then Givens QR of
// F V -> U and the singular values on the diagonal of R.
// Matrices are row-major a[r][c].
// ---------------------------------------------------------------------------
template <class R> struct M3 {
    R a[3][3];
};
template <class R> inline M3<R> mul(const M3<R>& A, const M3<R>& B) {
    M3<R> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            R s = 0;
            for (int k = 0; k < 3; k++) s += A.a[i][k] * B.a[k][j];
            C.a[i][j] = s;
        }
    return C;
}
template <class R> inline M3<R> transpose(const M3<R>& A) {
    M3<R> T;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) T.a[i][j] = A.a[j][i];
    return T;
}
template <class R> inline M3<R> eye3() {
    M3<R> I{};
    I.a[0][0] = I.a[1][1] = I.a[2][2] = R(1);
    return I;
}
template <class R> inline R det3(const M3<R>& A) {
    return A.a[0][0] * (A.a[1][1] * A.a[2][2] - A.a[1][2] * A.a[2][1]) -
           A.a[0][1] * (A.a[1][0] * A.a[2][2] - A.a[1][2] * A.a[2][0]) +
           A.a[0][2] * (A.a[1][0] * A.a[2][1] - A.a[1][1] * A.a[2][0]);
}

template <class R>
inline void svd3(const M3<R>& F, M3<R>& U, R S[3], M3<R>& V, int sweeps = 12) {
    // symmetric S = F^T F
    M3<R> A = mul(transpose(F), F);
    V = eye3<R>();
    for (int sw = 0; sw < sweeps; sw++) {
        R off = A.a[0][1] * A.a[0][1] + A.a[0][2] * A.a[0][2] + A.a[1][2] * A.a[1][2];
        if (off == R(0)) break;
        for (int pq = 0; pq < 3; pq++) {
            int p = pq == 2 ? 1 : 0;
            int q = pq == 0 ? 1 : 2;
            R apq = A.a[p][q];
            if (apq == R(0)) continue;
            R theta = (A.a[q][q] - A.a[p][p]) / (R(2) * apq);
            R t = (theta >= 0 ? R(1) : R(-1)) / (std::fabs(theta) + std::sqrt(theta * theta + R(1)));
            R c = R(1) / std::sqrt(t * t + R(1));
            R s = t * c;
            // A <- J^T A J with J = rotation in (p,q)
            for (int k = 0; k < 3; k++) {
                R akp = A.a[k][p], akq = A.a[k][q];
                A.a[k][p] = c * akp - s * akq;
                A.a[k][q] = s * akp + c * akq;
            }
            for (int k = 0; k < 3; k++) {
                R apk = A.a[p][k], aqk = A.a[q][k];
                A.a[p][k] = c * apk - s * aqk;
                A.a[q][k] = s * apk + c * aqk;
            }
            for (int k = 0; k < 3; k++) {
                R vkp = V.a[k][p], vkq = V.a[k][q];
                V.a[k][p] = c * vkp - s * vkq;
                V.a[k][q] = s * vkp + c * vkq;
            }
        }
    }
    // B = F V, sort columns by decreasing norm (swap with a sign flip keeps det V = +1)
    M3<R> B = mul(F, V);
    auto colnorm2 = [&](int j) { return B.a[0][j] * B.a[0][j] + B.a[1][j] * B.a[1][j] + B.a[2][j] * B.a[2][j]; };
    auto swapcols = [&](int i, int j) {
        for (int k = 0; k < 3; k++) {
            std::swap(B.a[k][i], B.a[k][j]);
            std::swap(V.a[k][i], V.a[k][j]);
            B.a[k][j] = -B.a[k][j];
            V.a[k][j] = -V.a[k][j];
        }
    };
    if (colnorm2(0) < colnorm2(1)) swapcols(0, 1);
    if (colnorm2(0) < colnorm2(2)) swapcols(0, 2);
    if (colnorm2(1) < colnorm2(2)) swapcols(1, 2);
    if (det3(V) < R(0)) {  // keep V a rotation
        for (int k = 0; k < 3; k++) { V.a[k][2] = -V.a[k][2]; B.a[k][2] = -B.a[k][2]; }
    }
    // Givens QR: B = U R, U a rotation, R upper triangular with R00, R11 >= 0
    U = eye3<R>();
    auto givens = [&](int r1, int r2, int col) {
        R a = B.a[r1][col], b = B.a[r2][col];
        R rr = std::sqrt(a * a + b * b);
        R c = R(1), s = R(0);
        if (rr > R(0)) { c = a / rr; s = b / rr; }
        for (int k = 0; k < 3; k++) {
            R x1 = B.a[r1][k], x2 = B.a[r2][k];
            B.a[r1][k] = c * x1 + s * x2;
            B.a[r2][k] = -s * x1 + c * x2;
        }
        // U <- U G^T
        for (int k = 0; k < 3; k++) {
            R u1 = U.a[k][r1], u2 = U.a[k][r2];
            U.a[k][r1] = c * u1 + s * u2;
            U.a[k][r2] = -s * u1 + c * u2;
        }
    };
    givens(0, 1, 0);
    givens(0, 2, 0);
    givens(1, 2, 1);
    S[0] = B.a[0][0];
    S[1] = B.a[1][1];
    S[2] = B.a[2][2];
}

// ---------------------------------------------------------------------------
// Prox operators (GPU semantics).
// ---------------------------------------------------------------------------
// tet: tetrahedral_constraint_device.cu:56-104 -> z = 1/2 (U V^T + F); F column j
// is z row j (zi_block[3j..3j+2]).
template <class R> inline void prox_tet(R z[9]) {
    M3<R> F;
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) F.a[i][j] = z[3 * j + i];
    M3<R> U, V;
    R S[3];
    svd3(F, U, S, V);
    M3<R> P = mul(U, transpose(V));
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) z[3 * j + i] = R(0.5) * (P.a[i][j] + F.a[i][j]);
}

// tri: triangle_constraint_device.cu:111-201 -> SVD of [F 0] (F = 3x2), P_ =
// U diag(.) V^T with the reference's pick of columns for tiny singular values.
template <class R> inline void prox_tri(R z[6]) {
    M3<R> A{};
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 3; i++) A.a[i][j] = z[3 * j + i];
    M3<R> U, V;
    R S[3];
    svd3(A, U, S, V);
    R d[3];
    int c0, c1;
    const R tiny = R(1e-8);
    if (std::fabs(S[0]) < tiny) { d[0] = 0; d[1] = 1; d[2] = 1; c0 = 1; c1 = 2; }
    else if (std::fabs(S[1]) < tiny) { d[0] = 1; d[1] = 0; d[2] = 1; c0 = 0; c1 = 2; }
    else { d[0] = 1; d[1] = 1; d[2] = 0; c0 = 0; c1 = 1; }
    M3<R> P;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            R s = 0;
            for (int k = 0; k < 3; k++) s += U.a[i][k] * d[k] * V.a[j][k];
            P.a[i][j] = s;
        }
    for (int i = 0; i < 3; i++) {
        z[i] = R(0.5) * (P.a[i][c0] + A.a[i][0]);
        z[3 + i] = R(0.5) * (P.a[i][c1] + A.a[i][1]);
    }
}

// bending: bending_constraint_device.cu:54-77
template <class R> inline void prox_bend(R z[3], R rest_norm) {
    R pn = std::sqrt((z[0] * z[0] + z[1] * z[1]) + z[2] * z[2]);
    R p[3] = {0, 0, 0};
    if (pn > R(1e-7)) {
        R sc = rest_norm / pn;
        p[0] = z[0] * sc; p[1] = z[1] * sc; p[2] = z[2] * sc;
    }
    for (int i = 0; i < 3; i++) z[i] = (z[i] + p[i]) / R(2);
}

}  // namespace orc
