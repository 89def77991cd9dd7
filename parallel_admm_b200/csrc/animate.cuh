// animate.cuh -- scripted static meshes (the reference's ScriptAnimator,
// src/solver/animator.cpp), applied on the device at the start of a substep.
//
// The reference computes the static rows on the host and copies them to the
// device every substep (admm_impl_gpu.cu:265-270).  Here the tracks live in
// HBM and two kernels of the step graph replace that: one thread advances the
// shared frame counter exactly as animate_all / animate_rigid / animate_points
// do (animator.cpp:81-90, 128-131, 185-203) and records each track's frame;
// then one thread per animated vertex writes its position into x0 and its
// velocity into v, which pre-integration turns into x = x0 and p = v.
#pragma once
#include "common.cuh"
#include "kernels.cuh"
#include "scene_dev.cuh"

namespace admm {

constexpr int kMaxTracks = 64;

struct TrackDev {
    int kind = 0;           // 0 rigid (pos + quat per frame), 1 points (one position per vertex and frame)
    int v0 = 0, v1 = 0;     // static vertex range
    int n_frames = 0;
    int first = 0;          // prefix of the animated vertices over the tracks
    const float4* pos = nullptr;   // rigid: [n_frames] translation
    const float4* quat = nullptr;  // rigid: [n_frames] (x, y, z, w)
    const float4* rest = nullptr;  // rigid: [v1 - v0] rest positions
    const float4* pts = nullptr;   // points: [n_frames][v1 - v0]
    float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // points: mesh rotation (row-major)
    float trans[3] = {0, 0, 0};                   // points: mesh translation
    float scale = 1.f;                            // points: mesh scale
};

struct AnimDev {
    int n_tracks = 0;
    int n_verts = 0;          // animated vertices over all tracks
    TrackDev* tracks = nullptr;
    int* counter = nullptr;   // the animator's m_curr_frame
    int* frame = nullptr;     // [n_tracks] frame read this substep
    int* moving = nullptr;    // [n_tracks] 1: velocity from the move, 0: zero velocity
};

// The frame bookkeeping of one animate_all call.  init: the call of
// ADMMImplGPU::init / reset (counter restarted, positions written in place,
// so the velocities come out zero).
__global__ void k_anim_advance(AnimDev a, int init) {
    ADMM_PDL_PROLOGUE();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int c = (init ? -1 : *a.counter) + 1;
    for (int t = 0; t < a.n_tracks; t++) {
        const TrackDev& tr = a.tracks[t];
        if (tr.kind == 0) c += 1;
        if (c >= tr.n_frames) {
            c = tr.n_frames;
            a.frame[t] = tr.n_frames - 1;
            a.moving[t] = 0;
        } else {
            a.frame[t] = tr.kind == 0 ? c - 1 : c;
            a.moving[t] = init ? 0 : 1;
        }
    }
    *a.counter = c;
}

// q * v for a unit quaternion q = (x, y, z, w): v + 2w (q x v) + 2 q x (q x v).
ADMM_DEV float4 quat_rotate(float4 q, float4 v) {
    const float ux = 2.f * (q.y * v.z - q.z * v.y);
    const float uy = 2.f * (q.z * v.x - q.x * v.z);
    const float uz = 2.f * (q.x * v.y - q.y * v.x);
    return f4(v.x + q.w * ux + (q.y * uz - q.z * uy), v.y + q.w * uy + (q.z * ux - q.x * uz),
              v.z + q.w * uz + (q.x * uy - q.y * ux));
}

__global__ void __launch_bounds__(kVertThreads) k_animate(DevScene s, AnimDev a) {
    ADMM_PDL_PROLOGUE();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n_verts) return;
    int t = 0;
    while (t + 1 < a.n_tracks && a.tracks[t + 1].first <= k) t++;
    const TrackDev& tr = a.tracks[t];
    const int j = k - tr.first, i = tr.v0 + j;
    const int f = a.frame[t];
    float4 x;
    if (tr.kind == 0) {
        const float4 r = quat_rotate(tr.quat[f], tr.rest[j]), p = tr.pos[f];
        x = f4(p.x + r.x, p.y + r.y, p.z + r.z);
    } else {
        const float4 q = tr.pts[(size_t)f * (tr.v1 - tr.v0) + j];
        const float qx = tr.scale * q.x, qy = tr.scale * q.y, qz = tr.scale * q.z;
        x = f4(tr.trans[0] + (tr.rot[0] * qx + tr.rot[1] * qy + tr.rot[2] * qz),
               tr.trans[1] + (tr.rot[3] * qx + tr.rot[4] * qy + tr.rot[5] * qz),
               tr.trans[2] + (tr.rot[6] * qx + tr.rot[7] * qy + tr.rot[8] * qz));
    }
    const float4 old = s.x0[i];
    s.v[i] = a.moving[t] ? f4((x.x - old.x) / s.dt, (x.y - old.y) / s.dt, (x.z - old.z) / s.dt) : f4(0.f, 0.f, 0.f);
    s.x0[i] = x;
}

}  // namespace admm
