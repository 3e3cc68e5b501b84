/* METIS stand-in: the reference includes metis.h but never partitions when it
 * runs serially (PartitionerSerial is only used with more than one rank).
 * Oracle test infrastructure only. */
#ifndef PG_SHIM_METIS_H
#define PG_SHIM_METIS_H
#include <stdint.h>
typedef int32_t idx_t;
typedef float real_t;
#define METIS_NOPTIONS 40
#define METIS_OK 1
#define METIS_OPTION_NUMBERING 17
#ifdef __cplusplus
extern "C" {
#endif
int METIS_SetDefaultOptions(idx_t* options);
int METIS_PartMeshDual(idx_t* ne, idx_t* nn, idx_t* eptr, idx_t* eind, idx_t* vwgt, idx_t* vsize,
                       idx_t* ncommon, idx_t* nparts, real_t* tpwgts, idx_t* options, idx_t* objval,
                       idx_t* epart, idx_t* npart);
int METIS_PartMeshNodal(idx_t* ne, idx_t* nn, idx_t* eptr, idx_t* eind, idx_t* vwgt, idx_t* vsize,
                        idx_t* nparts, real_t* tpwgts, idx_t* options, idx_t* objval,
                        idx_t* epart, idx_t* npart);
#ifdef __cplusplus
}
#endif
#endif
