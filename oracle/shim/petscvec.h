// Single-rank PETSc stand-in for the oracle build: everything lives in petsc.h.
#pragma once
#include <petsc.h>
