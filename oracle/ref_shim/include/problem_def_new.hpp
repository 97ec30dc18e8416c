// Stand-in for fr_sdg's include/problem_def_new.hpp (the Problem orchestrator and,
// through it, the PETSc TS/SNES glue of petsc_solver_impl.hpp), which
// problem_def.hpp includes last.  The checker library (oracle/ref_capi.cpp)
// restates the few callback bodies it needs instead, so this file is empty.
#pragma once
