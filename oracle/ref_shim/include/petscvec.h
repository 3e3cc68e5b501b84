/* Forwards to the single-rank PETSc stand-in (oracle test infrastructure). */
#ifndef PG_SHIM_PETSCVEC_H
#define PG_SHIM_PETSCVEC_H
#include "petsc_shim.h"
#endif
