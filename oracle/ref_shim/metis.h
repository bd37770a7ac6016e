/* TEST INFRASTRUCTURE ONLY — declarations standing in for METIS, written for this
 * project.  The reference calls METIS only to partition a mesh over MPI ranks; with one
 * rank and explicit host lists it is never reached, and this stand-in reports an error. */
#ifndef STEPS_SHIM_METIS_H
#define STEPS_SHIM_METIS_H
#include <stdint.h>
typedef int32_t idx_t;
typedef float real_t;
#define METIS_NOPTIONS 40
enum { METIS_OK = 1, METIS_ERROR = -4 };
enum {
    METIS_OPTION_PTYPE, METIS_OPTION_OBJTYPE, METIS_OPTION_CTYPE, METIS_OPTION_IPTYPE, METIS_OPTION_RTYPE,
    METIS_OPTION_DBGLVL, METIS_OPTION_NITER, METIS_OPTION_NCUTS, METIS_OPTION_SEED, METIS_OPTION_NO2HOP,
    METIS_OPTION_MINCONN, METIS_OPTION_CONTIG, METIS_OPTION_COMPRESS, METIS_OPTION_CCORDER, METIS_OPTION_PFACTOR,
    METIS_OPTION_NSEPS, METIS_OPTION_UFACTOR, METIS_OPTION_NUMBERING
};
enum { METIS_IPTYPE_GROW, METIS_IPTYPE_RANDOM, METIS_IPTYPE_EDGE, METIS_IPTYPE_NODE };
enum { METIS_OBJTYPE_CUT, METIS_OBJTYPE_VOL, METIS_OBJTYPE_NODE };
enum { METIS_DBG_INFO = 1, METIS_DBG_TIME = 2, METIS_DBG_CONTIGINFO = 4096 };
static inline int METIS_SetDefaultOptions(idx_t* o) {
    for (int i = 0; i < METIS_NOPTIONS; ++i) o[i] = -1;
    return METIS_OK;
}
static inline int METIS_PartMeshDual(idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, real_t*,
                                     idx_t*, idx_t*, idx_t*, idx_t*) {
    return METIS_ERROR;
}
#endif
