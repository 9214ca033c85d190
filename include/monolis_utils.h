/* monolis_utils.h
 *
 * The subset of the monolis_utils C interface that the monolis solver API
 * needs at its boundary: the communication-table struct MONOLIS_COM, the
 * logical constants and the self-communicator initialiser.
 *
 * monolis_utils is a git submodule of the reference (gitlab.com/mmlab_tsukuba/
 * monolis_utils) and its sources are not part of the reference tree, so the
 * field order of MONOLIS_COM below follows the fields that the reference's own
 * C code reads (wrapper/solver/monolis_solver_c.c:14-56,
 * wrapper/linalg/monolis_matvec_c.c:14-56): it is not pinned against the
 * submodule's header.
 */
#ifndef MONOLIS_UTILS_H
#define MONOLIS_UTILS_H

#ifdef __cplusplus
extern "C" {
#endif

#include <stdbool.h>

static const int MONOLIS_I_TRUE  = 1;
static const int MONOLIS_I_FALSE = 0;

/** Communication table of one rank (row partition with ghost nodes). */
typedef struct {
  int  comm;              /* MPI communicator handle (Fortran integer) */
  int  my_rank;
  int  comm_size;
  int  n_internal_vertex; /* N: rows owned by this rank */
  int  recv_n_neib;
  int* recv_neib_pe;
  int* recv_index;        /* recv_n_neib + 1 offsets */
  int* recv_item;         /* 0-based ghost node ids */
  int  send_n_neib;
  int* send_neib_pe;
  int* send_index;
  int* send_item;
} MONOLIS_COM;

/** Single-rank table: comm_size = 1, no neighbours. */
void monolis_com_initialize_by_self(MONOLIS_COM* com);

/** Frees the tables owned by com and resets it. */
void monolis_com_finalize(MONOLIS_COM* com);

#ifdef __cplusplus
}
#endif

#endif
