// prox.cuh -- per-constraint prox operators and the 3x3 SVD they use.
//
// Semantics follow the reference GPU prox functors:
//   tet  -- tetrahedral_constraint_device.cu:56-104: z = 1/2 (U V^T + F)
//   tri  -- triangle_constraint_device.cu:111-201:   SVD of [F 0], P = U S' V^T with
//           the reference's choice of S' and columns when a singular value is tiny
//   bend -- bending_constraint_device.cu:54-77:      z = 1/2 (z + rest * z/|z|)
//   pin  -- pin_constraint_device.cu:69-97:          z = pin position
// The SVD keeps the sign convention of the reference's svd (svd_fast3.cuh:37,
// after McAdams et al., UW-Madison TR1690, 2011): U and V are proper rotations,
// s1 >= s2 >= |s3|, only s3 may be negative -- so U V^T is the closest proper
// rotation.  It is computed here by cyclic Jacobi on F^T F with exact rotations
// (Golub & Van Loan, Alg. 8.5.2), column sorting, and a Givens QR of F V,
// which is accurate to float rounding.  (The reference's fixed-sweep
// approximate rotations reconstruct F only to about 2.5e-3 on well-conditioned
// inputs, so the two agree to that level, not to float rounding.)
#pragma once
#include "common.cuh"

namespace admm {

struct Mat3 {
    float a[3][3];  // row-major
};

ADMM_DEV void jacobi_rotate(float (&A)[3][3], float (&V)[3][3], int p, int q) {
    const float apq = A[p][q];
    if (apq == 0.f) return;
    const float theta = (A[q][q] - A[p][p]) / (2.f * apq);
    const float t = copysignf(1.f, theta) / (fabsf(theta) + sqrtf(fmaf(theta, theta, 1.f)));
    const float c = rsqrtf(fmaf(t, t, 1.f));
    const float s = t * c;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float akp = A[k][p], akq = A[k][q];
        A[k][p] = c * akp - s * akq;
        A[k][q] = s * akp + c * akq;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float apk = A[p][k], aqk = A[q][k];
        A[p][k] = c * apk - s * aqk;
        A[q][k] = s * apk + c * aqk;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float vkp = V[k][p], vkq = V[k][q];
        V[k][p] = c * vkp - s * vkq;
        V[k][q] = s * vkp + c * vkq;
    }
}

ADMM_DEV void givens_qr_step(float (&B)[3][3], float (&U)[3][3], int r1, int r2, int col) {
    const float a = B[r1][col], b = B[r2][col];
    const float rr2 = fmaf(a, a, b * b);
    float c = 1.f, s = 0.f;
    if (rr2 > 0.f) {
        const float inv = rsqrtf(rr2);
        c = a * inv;
        s = b * inv;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float x1 = B[r1][k], x2 = B[r2][k];
        B[r1][k] = c * x1 + s * x2;
        B[r2][k] = -s * x1 + c * x2;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float u1 = U[k][r1], u2 = U[k][r2];
        U[k][r1] = c * u1 + s * u2;
        U[k][r2] = -s * u1 + c * u2;
    }
}

// F = U diag(S) V^T.
ADMM_DEV void svd3(const float (&F)[3][3], float (&U)[3][3], float (&S)[3], float (&V)[3][3]) {
    float A[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            A[i][j] = F[0][i] * F[0][j] + F[1][i] * F[1][j] + F[2][i] * F[2][j];
            V[i][j] = (i == j) ? 1.f : 0.f;
        }
    // Jacobi converges quadratically; it stops once the off-diagonal mass is at the level of
    // FP32 rounding of the diagonal (|off| <= 1.2e-7 |diag|, squared: 1.4e-14), where further
    // rotations only move rounding noise (typically after 2-3 sweeps instead of all 6).
    for (int sweep = 0; sweep < 6; sweep++) {
        const float off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        const float dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1.4e-14f * dia || off == 0.f) break;
        jacobi_rotate(A, V, 0, 1);
        jacobi_rotate(A, V, 0, 2);
        jacobi_rotate(A, V, 1, 2);
    }
    float B[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) B[i][j] = F[i][0] * V[0][j] + F[i][1] * V[1][j] + F[i][2] * V[2][j];
    auto n2 = [&](int j) { return B[0][j] * B[0][j] + B[1][j] * B[1][j] + B[2][j] * B[2][j]; };
    auto swapcols = [&](int i, int j) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float t = B[k][i]; B[k][i] = B[k][j]; B[k][j] = -t;
            t = V[k][i]; V[k][i] = V[k][j]; V[k][j] = -t;
        }
    };
    if (n2(0) < n2(1)) swapcols(0, 1);
    if (n2(0) < n2(2)) swapcols(0, 2);
    if (n2(1) < n2(2)) swapcols(1, 2);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) U[i][j] = (i == j) ? 1.f : 0.f;
    givens_qr_step(B, U, 0, 1, 0);
    givens_qr_step(B, U, 0, 2, 0);
    givens_qr_step(B, U, 1, 2, 1);
    S[0] = B[0][0];
    S[1] = B[1][1];
    S[2] = B[2][2];
}

// z holds the constraint's rows; row j = column j of F.
ADMM_DEV void prox_tet(float (&z)[9]) {
    float F[3][3];
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) F[i][j] = z[3 * j + i];
    float U[3][3], V[3][3], S[3];
    svd3(F, U, S, V);
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float P = U[i][0] * V[j][0] + U[i][1] * V[j][1] + U[i][2] * V[j][2];
            z[3 * j + i] = 0.5f * (P + F[i][j]);
        }
}

ADMM_DEV void prox_tri(float (&z)[6]) {
    float A[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        A[i][0] = z[i];
        A[i][1] = z[3 + i];
        A[i][2] = 0.f;
    }
    float U[3][3], V[3][3], S[3];
    svd3(A, U, S, V);
    float d0 = 1.f, d1 = 1.f, d2 = 0.f;
    int c0 = 0, c1 = 1;
    if (fabsf(S[0]) < 1e-8f) { d0 = 0.f; d1 = 1.f; d2 = 1.f; c0 = 1; c1 = 2; }
    else if (fabsf(S[1]) < 1e-8f) { d0 = 1.f; d1 = 0.f; d2 = 1.f; c0 = 0; c1 = 2; }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const float p0 = U[i][0] * d0 * V[c0][0] + U[i][1] * d1 * V[c0][1] + U[i][2] * d2 * V[c0][2];
        const float p1 = U[i][0] * d0 * V[c1][0] + U[i][1] * d1 * V[c1][1] + U[i][2] * d2 * V[c1][2];
        z[i] = 0.5f * (p0 + A[i][0]);
        z[3 + i] = 0.5f * (p1 + A[i][1]);
    }
}

ADMM_DEV void prox_bend(float (&z)[3], float rest_norm) {
    const float pn = sqrtf(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
    float p0 = 0.f, p1 = 0.f, p2 = 0.f;
    if (pn > 1e-7f) {
        const float s = rest_norm / pn;
        p0 = z[0] * s; p1 = z[1] * s; p2 = z[2] * s;
    }
    z[0] = (z[0] + p0) * 0.5f;
    z[1] = (z[1] + p1) * 0.5f;
    z[2] = (z[2] + p2) * 0.5f;
}

}  // namespace admm
