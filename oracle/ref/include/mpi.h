/* Single-rank MPI interface used only to compile the reference's own sources into the
 * oracle harness (the container has no MPI).  Implementations: oracle/ref/mpi_stub.cpp.
 * Test infrastructure only. */
#pragma once
typedef int MPI_Comm; typedef int MPI_Datatype; typedef int MPI_Op; typedef int MPI_Request; typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_UNSIGNED 3
#define MPI_FLOAT 4
#define MPI_LONG 5
#define MPI_CHAR 6
#define MPI_DOUBLE_INT 7
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_MAXLOC 4
#define MPI_MINLOC 5
#define MPI_MAX_PROCESSOR_NAME 256
#ifdef __cplusplus
extern "C" {
#endif
int MPI_Init(int*, char***); int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm, int*); int MPI_Comm_size(MPI_Comm, int*);
int MPI_Barrier(MPI_Comm);
int MPI_Allreduce(void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Reduce(void*, void*, int, MPI_Datatype, MPI_Op, int, MPI_Comm);
int MPI_Isend(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*);
int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*);
int MPI_Send(void*, int, MPI_Datatype, int, int, MPI_Comm);
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*);
int MPI_Test(MPI_Request*, int*, MPI_Status*);
int MPI_Wait(MPI_Request*, MPI_Status*);
int MPI_Allgather(void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
int MPI_Allgatherv(void*, int, MPI_Datatype, void*, int*, int*, MPI_Datatype, MPI_Comm);
int MPI_Alltoall(void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm);
int MPI_Address(void*, MPI_Aint*);
int MPI_Type_struct(int, int*, MPI_Aint*, MPI_Datatype*, MPI_Datatype*);
int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype*);
int MPI_Type_commit(MPI_Datatype*); int MPI_Type_free(MPI_Datatype*);
double MPI_Wtime(void);
int MPI_Get_processor_name(char*, int*);
#ifdef __cplusplus
}
#endif
