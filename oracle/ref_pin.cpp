// ref_pin.cpp -- TEST INFRASTRUCTURE ONLY.  Compiles four of the reference's
// own headers, src/mutils/svd_fast3.cuh (3x3 SVD, McAdams et al. TR1690),
// src/mutils/dist_g.cuh (dcdPT / dcdEE narrow phase of the GPU backend) and
// src/mutils/distPT.h / distEE.h (the closest-point queries of the CPU backend),
// on the host against the stand-ins in oracle/ref_shim/, and exports them with a
// C ABI so the tests can pin the oracle's restatements to the reference's code.  The sources are read
// where they lie in the reference tree (see oracle/Makefile); nothing of them
// is copied into this repository.  Output goes to oracle/_ref/ only.
#include <cstdint>
#include <cstring>
#include "svd_fast3.cuh"
#include "dist_g.cuh"
#include "distEE.h"
#include "distPT.h"

extern "C" {

// F row-major 3x3 in; U, V row-major 3x3 and S[3] out.
void ref_svd3(const float* F, float* U, float* S, float* V) {
    svd(F[0], F[1], F[2], F[3], F[4], F[5], F[6], F[7], F[8],
        U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], U[8],
        S[0], S[1], S[2],
        V[0], V[1], V[2], V[3], V[4], V[5], V[6], V[7], V[8]);
}

static void pack(const Result<float>& r, float* out) {
    float o[11] = {r.distance, r.sqrDistance, r.barycentric[0], r.barycentric[1], r.barycentric[2],
                   r.closest[0][0], r.closest[0][1], r.closest[0][2],
                   r.closest[1][0], r.closest[1][1], r.closest[1][2]};
    std::memcpy(out, o, sizeof(o));
}

void ref_dcd_pt_f(const float* p, const float* t0, const float* t1, const float* t2, float* out) {
    Eigen::Vector3<float> P(p[0], p[1], p[2]), A(t0[0], t0[1], t0[2]), B(t1[0], t1[1], t1[2]), C(t2[0], t2[1], t2[2]);
    pack(dcdPT<float>(P, A, B, C), out);
}

void ref_dcd_ee_f(const float* p0, const float* p1, const float* q0, const float* q1, float* out) {
    Eigen::Vector3<float> P0(p0[0], p0[1], p0[2]), P1(p1[0], p1[1], p1[2]), Q0(q0[0], q0[1], q0[2]), Q1(q1[0], q1[1], q1[2]);
    pack(dcdEE<float>(P0, P1, Q0, Q1), out);
}

// CPU-backend closest points; out as for the above (edge-edge: parameters s, t
// in slots 2-3 and -2 in slot 4).
void ref_gt_pt_f(const float* p, const float* t0, const float* t1, const float* t2, float* out) {
    Eigen::Vector3<float> P(p[0], p[1], p[2]), A(t0[0], t0[1], t0[2]), B(t1[0], t1[1], t1[2]), C(t2[0], t2[1], t2[2]);
    ADU::DistPT<float> q;
    const auto r = q(P, A, B, C);
    float o[11] = {r.distance, r.sqrDistance, r.barycentric[0], r.barycentric[1], r.barycentric[2],
                   r.closest[0][0], r.closest[0][1], r.closest[0][2], r.closest[1][0], r.closest[1][1], r.closest[1][2]};
    std::memcpy(out, o, sizeof(o));
}

void ref_gt_ee_f(const float* p0, const float* p1, const float* q0, const float* q1, float* out) {
    Eigen::Vector3<float> P0(p0[0], p0[1], p0[2]), P1(p1[0], p1[1], p1[2]), Q0(q0[0], q0[1], q0[2]), Q1(q1[0], q1[1], q1[2]);
    ADU::DistEE<float> q;
    const auto r = q(P0, P1, Q0, Q1);
    float o[11] = {r.distance, r.sqrDistance, r.parameter[0], r.parameter[1], -2.f,
                   r.closest[0][0], r.closest[0][1], r.closest[0][2], r.closest[1][0], r.closest[1][1], r.closest[1][2]};
    std::memcpy(out, o, sizeof(o));
}

}
