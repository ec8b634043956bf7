/* oracle/shims/mpi.h -- single-rank stand-in for the MPI calls the reference programs make
 * (MPI_Init/Comm_rank/Comm_size/Get_processor_name/Barrier/Bcast/Allreduce/Finalize).
 * Test infrastructure: lets the reference sources build and run as one rank without MPICH. */
#ifndef SWD_SHIM_MPI_H
#define SWD_SHIM_MPI_H
#ifdef __cplusplus
extern "C" {
#endif
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_FLOAT 1
#define MPI_DOUBLE 2
#define MPI_INT 3
#define MPI_SUM 1
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_IN_PLACE ((void *)1)
int MPI_Init(int *argc, char ***argv);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Get_processor_name(char *name, int *len);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Finalize(void);
#ifdef __cplusplus
}
#endif
#endif
