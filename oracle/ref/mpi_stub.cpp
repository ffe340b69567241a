// Single-rank MPI for the oracle harness (test infrastructure).  Collectives copy the
// send buffer into the receive buffer; point-to-point calls never happen with one rank
// and abort if reached.
#include <mpi.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

struct DoubleInt {
    double d;
    int i;
};

static size_t tsize(MPI_Datatype t) {
    switch (t) {
        case MPI_INT: return sizeof(int);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_UNSIGNED: return sizeof(unsigned);
        case MPI_FLOAT: return sizeof(float);
        case MPI_LONG: return sizeof(long);
        case MPI_CHAR: return 1;
        case MPI_DOUBLE_INT: return sizeof(DoubleInt);
        default: return 0;
    }
}

static int unreachable(const char *f) {
    std::fprintf(stderr, "mpi_stub: %s called with a single rank\n", f);
    std::abort();
}

extern "C" {
int MPI_Init(int *, char ***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
int MPI_Allreduce(void *a, void *b, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (a != b) std::memmove(b, a, tsize(t) * n);
    return 0;
}
int MPI_Reduce(void *a, void *b, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (a != b) std::memmove(b, a, tsize(t) * n);
    return 0;
}
int MPI_Isend(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return unreachable("MPI_Isend"); }
int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return unreachable("MPI_Irecv"); }
int MPI_Send(void *, int, MPI_Datatype, int, int, MPI_Comm) { return unreachable("MPI_Send"); }
int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return unreachable("MPI_Recv"); }
int MPI_Test(MPI_Request *, int *flag, MPI_Status *) { *flag = 1; return 0; }
int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
int MPI_Allgather(void *a, int n, MPI_Datatype t, void *b, int, MPI_Datatype, MPI_Comm) {
    std::memmove(b, a, tsize(t) * n);
    return 0;
}
int MPI_Allgatherv(void *a, int n, MPI_Datatype t, void *b, int *, int *displs, MPI_Datatype, MPI_Comm) {
    std::memmove((char *)b + (displs ? displs[0] : 0) * tsize(t), a, tsize(t) * n);
    return 0;
}
int MPI_Alltoall(void *a, int n, MPI_Datatype t, void *b, int, MPI_Datatype, MPI_Comm) {
    std::memmove(b, a, tsize(t) * n);
    return 0;
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Address(void *p, MPI_Aint *a) { *a = (MPI_Aint)p; return 0; }
int MPI_Type_struct(int, int *, MPI_Aint *, MPI_Datatype *, MPI_Datatype *nt) { *nt = 100; return 0; }
int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype *nt) { *nt = 101; return 0; }
int MPI_Type_commit(MPI_Datatype *) { return 0; }
int MPI_Type_free(MPI_Datatype *) { return 0; }
double MPI_Wtime(void) { return double(std::clock()) / CLOCKS_PER_SEC; }
int MPI_Get_processor_name(char *n, int *len) {
    std::strcpy(n, "local");
    *len = 5;
    return 0;
}
}
