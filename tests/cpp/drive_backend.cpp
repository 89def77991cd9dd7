// TEST INFRASTRUCTURE ONLY.  Drives include/admm_b200_backend.hpp (the C++
// IADMMBackend adapter) with the reference's call order
// (src/app/app_initializer.cpp:142-228) on a scene read from a binary file
// written by tests/test_cpp_backend.py, and writes the positions after N steps.
//
//   drive_backend <scene.bin> <out.bin> [<contacts.bin>]
// With a third argument, the ICollisionDetector view (ADU::BVHB200) then detects on the
// positions after the steps and writes: count, max_slots, peak (int64 each), then
// max_slots points and max_slots normals (float32 x 3).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <memory>
#include <vector>

#include "admm_b200_backend.hpp"

namespace {
struct Reader {
    std::ifstream f;
    explicit Reader(const char* p) : f(p, std::ios::binary) {}
    template <class T>
    std::vector<T> arr() {
        int64_t n = 0;
        f.read(reinterpret_cast<char*>(&n), sizeof(n));
        std::vector<T> v((size_t)n);
        if (n) f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
        return v;
    }
};
}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: drive_backend scene.bin out.bin\n");
        return 2;
    }
    Reader r(argv[1]);
    auto I = r.arr<int32_t>();   // n_vert n_dyn n_rows tri_sr tet_sr bend_sr pin_sr admm dcd gs jac maxc contact nsteps lanes
    auto F = r.arr<float>();     // dt g mu kappa beta thickness
    auto verts = r.arr<float>(), mass = r.arr<float>();
    auto tri_inds = r.arr<int32_t>(); auto tri_binv = r.arr<float>(); auto tri_w = r.arr<float>();
    auto tet_inds = r.arr<int32_t>(); auto tet_binv = r.arr<float>(); auto tet_w = r.arr<float>();
    auto bend_off = r.arr<int32_t>(); auto bend_inds = r.arr<int32_t>(); auto bend_coef = r.arr<float>();
    auto bend_w = r.arr<float>();
    auto pin_inds = r.arr<int32_t>(); auto pin_pos = r.arr<float>(); auto pin_w = r.arr<float>();
    auto st = r.arr<int32_t>(), se = r.arr<int32_t>(), sv = r.arr<int32_t>();
    auto cw = r.arr<float>();
    const int n = I[0], nd = I[1], nrows = I[2], nsteps = I[13];

    // constraint objects as the reference's constraint factory produces them
    Solver::ConstraintsList cs;
    for (size_t c = 0; c < tri_w.size(); c++) {
        auto t = std::make_shared<TriangleConstraint>();
        t->type = 1; t->dim = 2; t->start_row = I[3] + 2 * (int)c; t->w = tri_w[c];
        t->inds = {tri_inds[3 * c], tri_inds[3 * c + 1], tri_inds[3 * c + 2]};
        for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) t->Binv.a[i][j] = tri_binv[4 * c + 2 * i + j];
        cs.push_back(t);
    }
    for (size_t c = 0; c < tet_w.size(); c++) {
        auto t = std::make_shared<TetrahedralConstraint>();
        t->type = 2; t->dim = 3; t->start_row = I[4] + 3 * (int)c; t->w = tet_w[c];
        t->inds = {tet_inds[4 * c], tet_inds[4 * c + 1], tet_inds[4 * c + 2], tet_inds[4 * c + 3]};
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) t->Binv.a[i][j] = tet_binv[9 * c + 3 * i + j];
        cs.push_back(t);
    }
    for (size_t c = 0; c < bend_w.size(); c++) {
        auto b = std::make_shared<BendingConstraint>();
        b->type = 3; b->dim = 1; b->start_row = I[5] + (int)c; b->w = bend_w[c];
        for (int k = bend_off[c]; k < bend_off[c + 1]; k++) {
            b->inds.push_back(bend_inds[k]);
            b->coeffs.push_back(bend_coef[k]);
        }
        cs.push_back(b);
    }
    Solver::ConstraintsList pins;
    for (size_t c = 0; c < pin_w.size(); c++) {
        auto p = std::make_shared<PinConstraint>();
        p->type = 4; p->dim = 1; p->start_row = I[6] + (int)c; p->w = pin_w[c];
        p->inds = {pin_inds[c]};
        for (int k = 0; k < 3; k++) p->pin_poistion.v[k] = pin_pos[3 * c + k];
        pins.push_back(p);
    }

    ADU::ADMMBackendB200 backend;
    backend.impl()->ell_lanes = I[14];
    Solver* inner = backend.as_solver();
    ADU::ADMMSolverConfig cfg;
    cfg.static_vert_begin = nd;
    cfg.admm_max_iter = I[7]; cfg.DCD_interval = I[8]; cfg.gs_max_iter = I[9]; cfg.global_jacobi_iter = I[10];
    cfg.enable_frictional_contact = I[12] != 0;
    cfg.g = F[1]; cfg.mu = F[2]; cfg.kappa = F[3]; cfg.beta = F[4];
    cfg.contact_w_list.v = cw;
    backend.apply_config(cfg);                                    // app_initializer.cpp:198
    inner->add_constraints(cs);                                   // :211
    std::vector<int> pin_ids(pin_inds.begin(), pin_inds.end());
    inner->addPins(pin_ids);                                      // :216
    inner->getConstraints().insert(inner->getConstraints().end(), pins.begin(), pins.end());  // :225
    backend.set_constraint_dim(nrows);                            // :227
    backend.finalize_constraints();                               // :228
    ContactParameter::set_thickness(F[5]);                        // :232
    auto mesh = std::make_shared<MeshData>();
    mesh->surface_tris.resize((int)st.size() / 3, 3); mesh->surface_tris.v = st;
    mesh->surface_edges.resize((int)se.size() / 2, 2); mesh->surface_edges.v = se;
    mesh->surface_vinds.v = sv;
    inner->prox_query = std::make_unique<ProximalQuery>(mesh, (size_t)I[11]);   // :234
    ADU::Matf_X3 V;
    V.resize(n, 3);
    V.v = verts;
    ADU::Vecf_X M;
    M.v = mass;
    try {
        inner->init(V, M, F[0]);                                  // :262
        backend.set_sync_to_host(true);                           // :267
        for (int s = 0; s < nsteps; s++) backend.step();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "drive_backend: %s\n", e.what());
        return 1;
    }
    std::ofstream o(argv[2], std::ios::binary);
    o.write(reinterpret_cast<const char*>(inner->m_vertices.data()), sizeof(float) * 3 * n);
    if (argc > 3) {
        try {
            ADU::BVHB200 det(backend);
            ADU::ICollisionDetector& cd = det;  // through the reference's contract
            cd.detect(inner->m_vertices);
            const int64_t head[3] = {(int64_t)cd.contact_count(), (int64_t)cd.max_slots(),
                                     (int64_t)cd.peak_contact_count()};
            const auto pts = cd.points();
            const auto nrm = cd.normals();
            std::ofstream c(argv[3], std::ios::binary);
            c.write(reinterpret_cast<const char*>(head), sizeof(head));
            for (const auto& p : pts) c.write(reinterpret_cast<const char*>(p.data()), sizeof(float) * 3);
            for (const auto& p : nrm) c.write(reinterpret_cast<const char*>(p.data()), sizeof(float) * 3);
        } catch (const std::exception& e) {
            std::fprintf(stderr, "drive_backend: %s\n", e.what());
            return 1;
        }
    }
    std::printf("steps %d contacts %zu\n", nsteps, inner->step_metrics.empty() ? 0 : inner->step_metrics.back().n_contacts);
    return 0;
}
