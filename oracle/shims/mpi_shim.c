/* oracle/shims/mpi_shim.c -- one-rank MPI: rank 0 of 1; Allreduce copies unless in place. */
#include <string.h>
#include "mpi.h"
static size_t type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }
int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
int MPI_Get_processor_name(char *name, int *len) { strcpy(name, "oracle"); *len = 6; return 0; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{ (void)buf; (void)count; (void)type; (void)root; (void)comm; return 0; }
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)op; (void)comm;
    if (send != MPI_IN_PLACE && send != recv) memcpy(recv, send, (size_t)count * type_size(type));
    return 0;
}
int MPI_Finalize(void) { return 0; }
