/* Forwards to the single-rank PETSc stand-in (oracle test infrastructure). */
#ifndef PG_SHIM_PETSC_H
#define PG_SHIM_PETSC_H
#include "petsc_shim.h"
#endif
