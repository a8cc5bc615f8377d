/*
 * Single-rank MPI implementation for the oracle build of the reference
 * (test infrastructure only; see mpi.h in this directory).
 */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static size_t type_size(MPI_Datatype t) {
    switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    case MPI_CHAR: return 1;
    case MPI_DOUBLE: return sizeof(double);
    default: return 0; /* struct types: never copied with one rank */
    }
}

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
    (void)argc; (void)argv; (void)required;
    *provided = MPI_THREAD_MULTIPLE;
    return 0;
}
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; fflush(stdout); exit(code); }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm *out) {
    (void)comm; (void)type; (void)key; (void)info; *out = 2; return 0;
}
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *out) {
    (void)comm; (void)key; *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : 3; return 0;
}
int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return 0; }
int MPI_Type_create_struct(int count, const int blocklengths[], const MPI_Aint offsets[],
                           const MPI_Datatype types[], MPI_Datatype *newtype) {
    (void)count; (void)blocklengths; (void)offsets; (void)types; *newtype = 100; return 0;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_free(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm) {
    (void)buf; (void)count; (void)t; (void)root; (void)comm; return 0;
}
int MPI_Scatterv(const void *sendbuf, const int sendcounts[], const int displs[], MPI_Datatype st,
                 void *recvbuf, int recvcount, MPI_Datatype rt, int root, MPI_Comm comm) {
    (void)st; (void)root; (void)comm; (void)recvcount;
    if (sendbuf && recvbuf && sendcounts)
        memcpy(recvbuf, (const char *)sendbuf + (size_t)displs[0] * type_size(rt),
               (size_t)sendcounts[0] * type_size(rt));
    return 0;
}
int MPI_Ireduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, int root,
                MPI_Comm comm, MPI_Request *req) {
    (void)op; (void)root; (void)comm;
    if (sendbuf != MPI_IN_PLACE && recvbuf && sendbuf)
        memcpy(recvbuf, sendbuf, (size_t)count * type_size(t));
    *req = 0;
    return 0;
}
int MPI_Ibarrier(MPI_Comm comm, MPI_Request *req) { (void)comm; *req = 0; return 0; }
int MPI_Testall(int count, MPI_Request reqs[], int *flag, MPI_Status statuses[]) {
    (void)count; (void)reqs; (void)statuses; *flag = 1; return 0;
}
double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
