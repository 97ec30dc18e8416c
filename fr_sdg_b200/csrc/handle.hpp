// handle.hpp -- the frsdg_handle behind the C ABI (include/frsdg.h), shared by the
// translation units that implement entry points on handles (capi.cu, batch.cu).
//
// The handle plays the role of the reference's PhysicsEvaluator + PetscSolver pair
// (physics_evaluator.hpp:158-318, petsc_solver_impl.hpp:444-755): it owns the reference
// element, the filter, the cached curved metrics, the boundary data and every workspace.
#pragma once
#include "../../include/frsdg.h"
#include "frsdg_internal.hpp"
#include "pplimit.hpp"
#include "setup_ops.hpp"
#include "stab.hpp"

#include <cuda_runtime.h>

struct frsdg_handle
{
    frsdg_config cfg{};
