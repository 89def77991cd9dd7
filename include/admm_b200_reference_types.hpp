// admm_b200_reference_types.hpp -- the reference types the C++ backend adapter
// (admm_b200_backend.hpp) is written against.  Inside the reference tree these
// are the reference's own headers; the adapter is compiled there, next to
// ADMMBackendGPU, with the reference's src/ on the include path.
#pragma once
#include "solver/solver.h"                     // Solver (src/solver/solver.h:22-193)
#include "solver/core/admm_backend.h"          // IADMMBackend (src/solver/core/admm_backend.h:15-41)
#include "solver/core/admm_config.h"           // ADMMSolverConfig (src/solver/core/admm_config.h:13-54)
#include "constraint/triangle_constraint.h"    // TriangleConstraint::Binv
#include "constraint/tetrahedral_constraint.h" // TetrahedralConstraint::Binv
#include "constraint/bending_constraint.h"     // BendingConstraint::coeffs, rest_mean_curvature_norm
#include "constraint/pin_constraint.h"         // PinConstraint::pin_poistion
#include "contact/contact_parameter.h"         // ContactParameter::get_thickness
#include "contact/narrow_phase.h"              // ProximalQuery::mesh (surface sets), max_collision_num
#include "contact/icollision_detector.h"       // ICollisionDetector (src/contact/icollision_detector.h:19-47)
