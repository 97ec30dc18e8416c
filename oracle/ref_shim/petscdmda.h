// petscdmda.h -- stand-in: see petsc_stub.h (test infrastructure of oracle/_ref).
#pragma once
#include "petsc_stub.h"
