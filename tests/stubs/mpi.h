/* Minimal declarations of the MPI calls the plugin shim uses (and MDI's
 * MDI_MPI_get_world_comm), for a compile check where MPI is not installed. */
#ifndef LIBERI_TEST_STUB_MPI_H
#define LIBERI_TEST_STUB_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_CHAR 3
#define MPI_BYTE 4
#define MPI_SUM 1
#define MPI_MIN 2
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MDI_MPI_get_world_comm(MPI_Comm *comm);
#endif
