// admm_b200_backend.hpp -- the B200 backend as an IADMMBackend (C++ host side).
//
// Drop-in for ADMMBackendGPU (src/solver/backend_gpu/admm_backend_gpu.h:13):
// the application keeps its call order (src/app/app_initializer.cpp:142-228)
//   apply_config -> add_constraints -> addPins -> set_constraint_dim ->
//   finalize_constraints -> init(verts, mass, dt) -> set_sync_to_host -> step()...
// and this header turns the reference's constraint objects into the plain
// arrays of the C ABI (include/admm_b200.h) -- the job convert_constraint2device
// and precompute do for the reference GPU backend (admm_impl_gpu.cu:61-254) --
// then drives libadmm_b200.so.  Errors from the C ABI become std::runtime_error
// (the reference exits the process on CUDA errors, cuda_tools.cuh:37-46).
//
// Header-only; compile it where the reference headers are on the include path
// (admm_b200_reference_types.hpp) and link libadmm_b200.so.
#pragma once
#include <algorithm>
#include <array>
#include <chrono>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "admm_b200.h"
#include <admm_b200_reference_types.hpp>  // the reference headers, found through the include path

namespace ADU {

class ADMMInnerB200 : public Solver {
public:
    ADMMSolverConfig cfg;
    int n_rows = 0;
    bool finalized = false;
    bool sync_to_host = true;
    int device = 0;
    int ell_lanes = 0;    // 0 = autotuned
    int jacobi_mode = 0;  // 0 = autotuned
    int broad_phase = 0;  // 0 = default (uniform grid)
    int global_solver = 0;  // 0 = Jacobi as the reference
    int pcg_iter = 0;
    int query_lanes = 0;  // 0 = chosen from the number of DCD queries
    int contact_semantics = 0;  // 1 = the CPU backend's contact predicates (ProximalQuery)
    int backend_semantics = 0;  // 1 = the CPU backend's solver (damping, S_c, serial Gauss-Seidel contact)

    ~ADMMInnerB200() override {
        if (h_) admm_b200_destroy(h_);
    }

    // Solver::init(verts, mass, dt) sets m_vertices, m_M_vec, m_dt, m_nVert and
    // calls this (solver.h:66-90); the reference GPU backend precomputes here.
    void init() override {
        if (!finalized) throw std::runtime_error("ADMMBackendB200: init before finalize_constraints");
        build_description();
        AdmmB200* h = nullptr;
        const int rc = admm_b200_create(&desc_, device, &h);
        if (rc != ADMM_OK) throw std::runtime_error(std::string("admm_b200_create: ") + admm_b200_errstr(rc));
        h_ = h;  // the library copied everything it needs from desc_
    }

    void step() override {
        const auto t0 = std::chrono::steady_clock::now();
        AdmmStepStats st{};
        const int rc = admm_b200_step(h_, 1, &st);
        if (rc != ADMM_OK && rc != ADMM_ERR_CONTACT_OVERFLOW && rc != ADMM_ERR_STACK_OVERFLOW)
            throw std::runtime_error(std::string("admm_b200_step: ") + admm_b200_errstr(rc) + " / " +
                                     admm_b200_last_error(h_));
        if (sync_to_host) pull_state();
        step_cnt++;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        step_metrics.push_back({step_cnt, ms, (size_t)st.n_contacts});
        last_stats = st;
    }

    // ADMMImplGPU::reset (admm_impl_gpu.cu:151-155): back to ini_verts, zero
    // velocity and duals.
    void reset(const Matf_X3& ini_verts, bool /*need_precompute*/ = false) override {
        check(admm_b200_reset(h_), "admm_b200_reset");
        if (ini_verts.rows() == m_nVert) {
            std::vector<float> zero((size_t)m_nVert * 3, 0.f);
            check(admm_b200_set_state(h_, ini_verts.data(), zero.data(), m_nVert), "admm_b200_set_state");
        }
        pull_state();
    }

    void pull_state() {
        check(admm_b200_get_state(h_, m_vertices.data(), m_velocities.data(), m_nVert), "admm_b200_get_state");
    }

    AdmmB200* handle() { return h_; }
    AdmmStepStats last_stats{};

private:
    AdmmB200* h_ = nullptr;
    AdmmB200Desc desc_{};
    struct Arrays {
        std::vector<int32_t> fixed, tri_inds, tet_inds, bend_off, bend_inds, pin_inds, st, se, sv;
        std::vector<float> tri_binv, tri_w, tet_binv, tet_w, bend_coef, bend_rest, bend_w, pin_pos, pin_w, cw;
    } a_;

    static void check(int rc, const char* what) {
        if (rc != ADMM_OK) throw std::runtime_error(std::string(what) + ": " + admm_b200_errstr(rc));
    }

    // convert_constraint2device (admm_impl_gpu.cu:61-96): one contiguous block of
    // rows per constraint type, start row of the first constraint of each type.
    void build_description() {
        Arrays& a = a_;
        a = Arrays{};
        int sr[5] = {-1, -1, -1, -1, -1}, cnt[5] = {0, 0, 0, 0, 0};
        const int dims[5] = {0, 2, 3, 1, 1};
        a.bend_off.push_back(0);
        for (const auto& ct : m_constraints) {
            const int t = ct->type;
            if (t < 1 || t > 4) throw std::runtime_error("ADMMBackendB200: unsupported constraint type");
            if (sr[t] < 0) sr[t] = ct->start_row;
            if (ct->start_row != sr[t] + dims[t] * cnt[t])
                throw std::runtime_error("ADMMBackendB200: rows of one constraint type must be contiguous");
            cnt[t]++;
            if (t == 1) {
                auto* c = static_cast<const TriangleConstraint*>(ct.get());
                for (int k = 0; k < 3; k++) a.tri_inds.push_back(c->inds[k]);
                for (int r = 0; r < 2; r++)
                    for (int q = 0; q < 2; q++) a.tri_binv.push_back(c->Binv(r, q));
                a.tri_w.push_back(c->w);
            } else if (t == 2) {
                auto* c = static_cast<const TetrahedralConstraint*>(ct.get());
                for (int k = 0; k < 4; k++) a.tet_inds.push_back(c->inds[k]);
                for (int r = 0; r < 3; r++)
                    for (int q = 0; q < 3; q++) a.tet_binv.push_back(c->Binv(r, q));
                a.tet_w.push_back(c->w);
            } else if (t == 3) {
                auto* c = static_cast<const BendingConstraint*>(ct.get());
                for (size_t k = 0; k < c->inds.size(); k++) {
                    a.bend_inds.push_back(c->inds[k]);
                    a.bend_coef.push_back(c->coeffs[k]);
                }
                a.bend_off.push_back((int32_t)a.bend_inds.size());
                a.bend_rest.push_back(c->rest_mean_curvature_norm);
                a.bend_w.push_back(c->w);
            } else {
                auto* c = static_cast<const PinConstraint*>(ct.get());
                a.pin_inds.push_back(c->inds[0]);
                for (int k = 0; k < 3; k++) a.pin_pos.push_back(c->pin_poistion(k));
                a.pin_w.push_back(c->w);
            }
        }
        a.fixed.assign(m_nVert, 0);
        for (int p : m_pin_inds_set)
            if (p >= 0 && p < m_nVert) a.fixed[p] = 1;
        AdmmB200Desc& d = desc_;
        d = AdmmB200Desc{};
        d.abi_version = ADMM_B200_ABI_VERSION;
        d.n_vert = m_nVert;
        d.n_dyn = cfg.static_vert_begin > 0 ? cfg.static_vert_begin : m_nVert;
        d.n_rows = n_rows;
        d.x0 = m_vertices.data();
        d.v0 = m_velocities.data();
        d.mass = m_M_vec.data();
        d.is_fixed = a.fixed.data();
        d.n_tri = cnt[1]; d.tri_start_row = sr[1] < 0 ? 0 : sr[1];
        d.tri_inds = a.tri_inds.data(); d.tri_binv = a.tri_binv.data(); d.tri_w = a.tri_w.data();
        d.n_tet = cnt[2]; d.tet_start_row = sr[2] < 0 ? 0 : sr[2];
        d.tet_inds = a.tet_inds.data(); d.tet_binv = a.tet_binv.data(); d.tet_w = a.tet_w.data();
        d.n_bend = cnt[3]; d.bend_start_row = sr[3] < 0 ? 0 : sr[3];
        d.bend_offsets = a.bend_off.data(); d.bend_inds = a.bend_inds.data(); d.bend_coeffs = a.bend_coef.data();
        d.bend_rest_norm = a.bend_rest.data(); d.bend_w = a.bend_w.data();
        d.n_pin = cnt[4]; d.pin_start_row = sr[4] < 0 ? 0 : sr[4];
        d.pin_inds = a.pin_inds.data(); d.pin_pos = a.pin_pos.data(); d.pin_w = a.pin_w.data();
        const bool contact = cfg.enable_frictional_contact && prox_query && prox_query->mesh;
        if (contact) {
            const auto& mesh = *prox_query->mesh;
            a.st.assign(mesh.surface_tris.data(), mesh.surface_tris.data() + mesh.surface_tris.rows() * 3);
            a.se.assign(mesh.surface_edges.data(), mesh.surface_edges.data() + mesh.surface_edges.rows() * 2);
            a.sv.assign(mesh.surface_vinds.data(), mesh.surface_vinds.data() + mesh.surface_vinds.rows());
            a.cw.assign(cfg.contact_w_list.data(), cfg.contact_w_list.data() + cfg.contact_w_list.rows());
        }
        d.n_surf_tri = (int32_t)(a.st.size() / 3);
        d.n_surf_edge = (int32_t)(a.se.size() / 2);
        d.n_surf_vert = (int32_t)a.sv.size();
        d.surf_tris = a.st.data(); d.surf_edges = a.se.data(); d.surf_verts = a.sv.data();
        d.contact_w = contact ? a.cw.data() : nullptr;
        d.dt = m_dt;
        d.g = cfg.g;
        d.mu = cfg.mu;
        d.kappa = cfg.kappa;
        d.beta = cfg.beta;
        d.thickness = ContactParameter::get_thickness();
        d.admm_max_iter = cfg.admm_max_iter;
        d.dcd_interval = cfg.DCD_interval;
        d.gs_max_iter = cfg.gs_max_iter;
        d.jacobi_iter = cfg.global_jacobi_iter;
        d.max_contacts = prox_query ? (int32_t)prox_query->max_collision_num : 100000;
        d.enable_contact = contact ? 1 : 0;
        d.warmstart_ue = cfg.warmstart_Ue ? 1 : 0;
        d.warmstart_uc = cfg.warmstart_Uc ? 1 : 0;
        d.residual_tol = 0.f;
        d.residual_check_every = 0;
        d.bvh_refit = 1;
        d.ell_lanes = ell_lanes;
        d.jacobi_mode = jacobi_mode;
        d.broad_phase = broad_phase;
        d.global_solver = global_solver;
        d.pcg_iter = pcg_iter;
        d.query_lanes = query_lanes;
        d.contact_semantics = contact_semantics;
        d.backend_semantics = backend_semantics;
        d.damp_k_L = (float)cfg.damp_k_L;  // ADMMSolverConfig (admm_config.h:52-53)
        d.damp_k_M = (float)cfg.damp_k_M;
    }
};

// IADMMBackend over the B200 library (the counterpart of ADMMBackendGPU).
class ADMMBackendB200 : public IADMMBackend {
public:
    explicit ADMMBackendB200(int device = 0) : impl_(std::make_unique<ADMMInnerB200>()) { impl_->device = device; }

    void precompute() override {}  // assembly happens in init, when mass and dt are known
    void step() override { impl_->step(); }
    Solver* as_solver() override { return impl_.get(); }
    void apply_config(const ADMMSolverConfig& cfg) override { impl_->cfg = cfg; }
    void finalize_constraints() override { impl_->finalized = true; }
    void set_constraint_dim(int n) override { impl_->n_rows = n; }
    void set_sync_to_host(bool enabled) override { impl_->sync_to_host = enabled; }

    ADMMInnerB200* impl() { return impl_.get(); }

private:
    std::unique_ptr<ADMMInnerB200> impl_;
};

// ICollisionDetector over the backend's handle: the counterpart of BVH_GPU
// (src/contact/collision_detection_cuda.h:45) for the contract of
// src/contact/icollision_detector.h:19-47.  A view, not an owner: the handle (and its
// contact buffers) belongs to the backend and exists from init() on, so calls before
// init() throw.  detect() uploads host positions and runs the library's detection
// (broad phase + narrow phase + contact conversion) on the handle; points() and
// normals() return exactly max_slots() rows, the rows past contact_count() zero
// (the GUI registers point clouds of max_slots() points, icollision_detector.h:36-44).
class BVHB200 : public ICollisionDetector {
public:
    explicit BVHB200(ADMMBackendB200& backend) : backend_(backend) {}

    void detect(const Matf_X3& pos) override {
        int cnt = 0;
        const int rc = admm_b200_detect_host(h(), pos.data(), pos.rows(), &cnt);
        if (rc != ADMM_OK && rc != ADMM_ERR_CONTACT_OVERFLOW && rc != ADMM_ERR_STACK_OVERFLOW)
            throw std::runtime_error(std::string("admm_b200_detect_host: ") + admm_b200_errstr(rc));
    }
    size_t contact_count() const override {
        int c = 0;
        check(admm_b200_contact_count(h(), &c), "admm_b200_contact_count");
        return (size_t)c;
    }
    size_t max_slots() const override {
        int c = 0;
        check(admm_b200_max_slots(h(), &c), "admm_b200_max_slots");
        return (size_t)c;
    }
    size_t peak_contact_count() const override {
        int c = 0;
        check(admm_b200_peak_contact_count(h(), &c), "admm_b200_peak_contact_count");
        return (size_t)c;
    }
    std::vector<std::array<float, 3>> points() override { return rows(true); }
    std::vector<std::array<float, 3>> normals() override { return rows(false); }
    void clear() override { check(admm_b200_clear_contacts(h()), "admm_b200_clear_contacts"); }

private:
    ADMMBackendB200& backend_;

    AdmmB200* h() const {
        AdmmB200* p = backend_.impl()->handle();
        if (!p) throw std::runtime_error("BVHB200: the backend has no handle before init()");
        return p;
    }
    static void check(int rc, const char* what) {
        if (rc != ADMM_OK) throw std::runtime_error(std::string(what) + ": " + admm_b200_errstr(rc));
    }
    std::vector<std::array<float, 3>> rows(bool pts) {
        const size_t slots = max_slots();
        std::vector<std::array<float, 3>> out(slots, std::array<float, 3>{0.f, 0.f, 0.f});
        const size_t n = std::min(contact_count(), slots);
        if (n == 0) return out;
        std::vector<float> buf(3 * n);
        int got = 0;
        const int rc = pts ? admm_b200_contacts(h(), nullptr, nullptr, nullptr, buf.data(), nullptr, (int)n, &got)
                           : admm_b200_contacts(h(), nullptr, nullptr, buf.data(), nullptr, nullptr, (int)n, &got);
        if (rc != ADMM_OK && rc != ADMM_ERR_CONTACT_OVERFLOW) check(rc, "admm_b200_contacts");
        for (size_t i = 0; i < n && i < (size_t)got; i++) out[i] = {buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]};
        return out;
    }
};

}  // namespace ADU
