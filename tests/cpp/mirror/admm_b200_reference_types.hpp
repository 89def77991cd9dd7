// TEST INFRASTRUCTURE ONLY.  A minimal, Eigen-free stand-in for the reference
// types that include/admm_b200_backend.hpp uses, with the same names, members
// and virtual functions (src/solver/solver.h, src/solver/core/admm_backend.h,
// src/solver/core/admm_config.h, src/constraint/*_constraint.h,
// src/contact/contact_parameter.h, src/contact/narrow_phase.h,
// src/contact/icollision_detector.h), so the adapter
// compiles and runs here without the reference's dependencies.  Put this
// directory before include/ on the include path.
#pragma once
#include <array>
#include <cstddef>
#include <memory>
#include <unordered_set>
#include <vector>

namespace ADU {
using Real = float;
template <class T, int C>
struct RowMat {  // row-major N x C, like Eigen::Matrix<T, Dynamic, C, RowMajor>
    std::vector<T> v;
    int r = 0;
    int rows() const { return r; }
    T* data() { return v.data(); }
    const T* data() const { return v.data(); }
    void resize(int rr, int) { r = rr; v.assign((size_t)rr * C, T(0)); }
    T& operator()(int i, int j) { return v[(size_t)i * C + j]; }
};
template <class T>
struct Vec {
    std::vector<T> v;
    int rows() const { return (int)v.size(); }
    T* data() { return v.data(); }
    const T* data() const { return v.data(); }
    void resize(int n) { v.assign(n, T(0)); }
    T& operator()(int i) { return v[i]; }
};
using Matf_X3 = RowMat<float, 3>;
using Mati_X3 = RowMat<int, 3>;
using Mati_X2 = RowMat<int, 2>;
using Vecf_X = Vec<float>;
using Veci_X = Vec<int>;
template <int R, int C>
struct Fixed {
    float a[R][C] = {};
    float operator()(int i, int j) const { return a[i][j]; }
};
using Matf_22 = Fixed<2, 2>;
using Matf_33 = Fixed<3, 3>;
struct Vecf_3 {
    float v[3] = {0, 0, 0};
    float operator()(int i) const { return v[i]; }
};

struct ADMMSolverConfig {
    int static_mesh_id_begin{};
    int static_vert_begin{};
    int admm_max_iter{25};
    int DCD_interval{5};
    int gs_max_iter{10};
    int global_jacobi_iter{20};
    bool warmstart_Ue{true};
    bool warmstart_Uc{true};
    Real g{0.98f};
    bool enable_frictional_contact{true};
    Real mu{0.5f};
    Real kappa{1e6f};
    Real beta{1e5f};
    Real damp_k_L{1e-4f};
    Real damp_k_M{0.0f};
    Vecf_X contact_w_list;
    Vecf_X contact_w_inv_list;
};
}  // namespace ADU

namespace ADU {
// src/contact/icollision_detector.h:19-47 (host-facing collision-detection contract)
class ICollisionDetector {
public:
    virtual ~ICollisionDetector() = default;
    virtual void detect(const Matf_X3& pos) = 0;
    virtual size_t contact_count() const = 0;
    virtual size_t max_slots() const = 0;
    virtual size_t peak_contact_count() const = 0;
    virtual std::vector<std::array<float, 3>> points() = 0;
    virtual std::vector<std::array<float, 3>> normals() = 0;
    virtual void clear() = 0;
};
}  // namespace ADU

class Constraint {
public:
    std::vector<int> inds;
    int type = 0;
    ADU::Real k{}, w{};
    int dim = 0, start_row{}, global_m{};
    virtual ~Constraint() = default;
};
class TriangleConstraint : public Constraint { public: ADU::Matf_22 Binv; };
class TetrahedralConstraint : public Constraint { public: ADU::Matf_33 Binv; };
class BendingConstraint : public Constraint {
public:
    std::vector<ADU::Real> coeffs;
    ADU::Real rest_mean_curvature_norm{};
};
class PinConstraint : public Constraint { public: ADU::Vecf_3 pin_poistion; };

class ContactParameter {
public:
    static ADU::Real& thickness() { static ADU::Real t = 0.005f; return t; }
    static ADU::Real get_thickness() { return thickness(); }
    static void set_thickness(ADU::Real t) { thickness() = t; }
};

struct MeshData {
    ADU::Mati_X3 surface_tris;
    ADU::Mati_X2 surface_edges;
    ADU::Veci_X surface_vinds;
};
class ProximalQuery {
public:
    ProximalQuery(std::shared_ptr<MeshData> m, size_t n) : mesh(std::move(m)), max_collision_num(n) {}
    std::shared_ptr<MeshData> mesh;
    const size_t max_collision_num;
};

class Solver {
public:
    struct StepMetrics {
        size_t frame{};
        double step_ms{};
        size_t n_contacts{};
    };
    std::vector<StepMetrics> step_metrics;
    size_t step_cnt = 0;
    std::unique_ptr<ProximalQuery> prox_query;
    using ConstraintsList = std::vector<std::shared_ptr<Constraint>>;
    virtual ~Solver() = default;
    virtual void init() {}
    virtual void init(const ADU::Matf_X3& verts, const ADU::Vecf_X& mass, ADU::Real dt) {
        m_vertices = verts;
        m_velocities.resize(verts.rows(), 3);
        m_M_vec = mass;
        m_dt = dt;
        m_nVert = verts.rows();
        init();
    }
    virtual void reset(const ADU::Matf_X3&, bool = false) {}
    virtual void step() {}
    virtual void add_constraints(const ConstraintsList& c) { m_constraints.insert(m_constraints.end(), c.begin(), c.end()); }
    virtual void addPins(const std::vector<int>& p) { m_pin_inds_set.insert(p.begin(), p.end()); }
    ConstraintsList& getConstraints() { return m_constraints; }
    ADU::Matf_X3 m_vertices, m_velocities;
    ADU::Vecf_X m_M_vec;
    std::unordered_set<int> m_pin_inds_set;
    ConstraintsList m_constraints;
    ADU::Real m_dt{};
    int m_nVert{};
};

namespace ADU {
struct IADMMBackend {
    virtual void precompute() = 0;
    virtual void step() = 0;
    virtual ::Solver* as_solver() = 0;
    virtual ~IADMMBackend() = default;
    virtual void apply_config(const ADMMSolverConfig& cfg) = 0;
    virtual void finalize_constraints() = 0;
    virtual void set_constraint_dim(int n) = 0;
    virtual void set_sync_to_host(bool) {}
};
}  // namespace ADU
