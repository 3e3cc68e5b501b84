/* Forwards to the single-rank PETSc stand-in (oracle test infrastructure). */
#ifndef PG_SHIM_PETSCMAT_H
#define PG_SHIM_PETSCMAT_H
#include "petsc_shim.h"
#endif
