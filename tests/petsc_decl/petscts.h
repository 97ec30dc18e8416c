/* declaration-only stand-in, see petsc_decl.h */
#pragma once
#include "petsc_decl.h"
