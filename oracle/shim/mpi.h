/*
 * Single-rank stand-in for the MPI API, used ONLY to compile the reference
 * NISE program from its own unmodified sources as a test oracle (oracle/_ref).
 *
 * Test infrastructure: nothing in the product links this.  Every call
 * behaves as MPI would with exactly one rank: broadcasts and scatters are
 * local copies, reductions with MPI_IN_PLACE are no-ops, requests complete
 * immediately.  Names and signatures follow the MPI-3 standard.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef ptrdiff_t MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_UNDEFINED (-32766)
#define MPI_INFO_NULL 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_SUM 1
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)-1)

/* Datatype handles encode their size in bytes (struct types are registered). */
#define MPI_INT 4
#define MPI_FLOAT 5
#define MPI_CHAR 6
#define MPI_DOUBLE 7

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm *out);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *out);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Type_create_struct(int count, const int blocklengths[], const MPI_Aint offsets[],
                           const MPI_Datatype types[], MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Scatterv(const void *sendbuf, const int sendcounts[], const int displs[], MPI_Datatype st,
                 void *recvbuf, int recvcount, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Ireduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, int root,
                MPI_Comm comm, MPI_Request *req);
int MPI_Ibarrier(MPI_Comm comm, MPI_Request *req);
int MPI_Testall(int count, MPI_Request reqs[], int *flag, MPI_Status statuses[]);
double MPI_Wtime(void);

#endif
