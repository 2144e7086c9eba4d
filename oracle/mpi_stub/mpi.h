/* Single-process stand-in for the few MPI names NEP3_CPU mentions.  Only its
 * charge (Ewald/PPPM) paths call MPI_Allreduce; the NEP4/NEP5/ZBL paths the
 * oracle drives never reach them.  TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H
#include <string.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_DOUBLE 0
#define MPI_SUM 0
static inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype type,
                                MPI_Op op, MPI_Comm comm)
{
  (void)type; (void)op; (void)comm;
  if (in != out) memcpy(out, in, sizeof(double) * (size_t)count);
  return 0;
}
#endif
