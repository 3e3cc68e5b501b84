/* Forwards to the single-rank PETSc stand-in (oracle test infrastructure). */
#ifndef PG_SHIM_PETSCIS_H
#define PG_SHIM_PETSCIS_H
#include "petsc_shim.h"
#endif
