/* Single-rank stand-in for an MPI implementation (TEST INFRASTRUCTURE ONLY).
 *
 * The reference's parallel classes (ParCSRMatrix, ParMultilevel, PCG, ...)
 * include <mpi.h>; no MPI library exists on the build machine or the GPU
 * machine.  This header and mpi_stub.cpp provide the subset of the MPI-3 C
 * interface those sources call, for exactly one process (COMM_WORLD has size
 * 1, every communicator derived from it too):
 *   - collectives copy the send buffer to the receive buffer (MPI_IN_PLACE
 *     leaves it where it is), so every reduction is the identity;
 *   - point-to-point messages can only go to rank 0 itself: a send copies
 *     the data into a queue kept per communicator, and a receive, probe or
 *     wait takes the oldest queued message whose source and tag match
 *     (MPI's non-overtaking order).  A blocking receive or probe that finds
 *     nothing would wait forever in a real MPI; here it aborts with a message.
 * Handles (communicators, groups, datatypes, operations, requests) are ints.
 * The names and argument lists follow the MPI standard, which is what makes
 * the reference compile unchanged against this file.
 */
#ifndef RAPTOR_ORACLE_MPI_STUB_H
#define RAPTOR_ORACLE_MPI_STUB_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;

typedef struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    long long stub_bytes; /* size of the matched message in bytes */
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15

#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_SELF ((MPI_Comm)2)
#define MPI_GROUP_NULL ((MPI_Group)0)
#define MPI_GROUP_EMPTY ((MPI_Group)-1)
#define MPI_REQUEST_NULL ((MPI_Request)0)

/* datatypes: the value encodes nothing; sizes come from mpi_stub_type_size */
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)2)
#define MPI_INT ((MPI_Datatype)3)
#define MPI_LONG ((MPI_Datatype)4)
#define MPI_UNSIGNED ((MPI_Datatype)5)
#define MPI_FLOAT ((MPI_Datatype)6)
#define MPI_DOUBLE ((MPI_Datatype)7)
#define MPI_DOUBLE_INT ((MPI_Datatype)8)
#define MPI_PACKED ((MPI_Datatype)9)
#define MPI_LONG_LONG ((MPI_Datatype)10)
#define MPI_UNSIGNED_LONG ((MPI_Datatype)11)

#define MPI_OP_NULL ((MPI_Op)0)
#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_PROD ((MPI_Op)4)
#define MPI_BOR ((MPI_Op)5)
#define MPI_BAND ((MPI_Op)6)
#define MPI_LOR ((MPI_Op)7)
#define MPI_LAND ((MPI_Op)8)
#define MPI_MAXLOC ((MPI_Op)9)
#define MPI_MINLOC ((MPI_Op)10)

#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_PROC_NULL (-2)
#define MPI_UNDEFINED (-32766)

#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

int MPI_Init(int* argc, char*** argv);
int MPI_Initialized(int* flag);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);

int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_group(MPI_Comm comm, MPI_Group* group);
int MPI_Comm_create_group(MPI_Comm comm, MPI_Group group, int tag, MPI_Comm* newcomm);
int MPI_Group_incl(MPI_Group group, int n, const int ranks[], MPI_Group* newgroup);
int MPI_Group_free(MPI_Group* group);

int MPI_Barrier(MPI_Comm comm);
int MPI_Ibarrier(MPI_Comm comm, MPI_Request* request);
int MPI_Bcast(void* buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype,
                  MPI_Op op, MPI_Comm comm);
int MPI_Iallreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype,
                   MPI_Op op, MPI_Comm comm, MPI_Request* request);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype,
               MPI_Op op, int root, MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
               int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int recvcounts[], const int displs[], MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                   const int recvcounts[], const int displs[], MPI_Datatype recvtype,
                   MPI_Comm comm);

int MPI_Send(const void* buf, int count, MPI_Datatype datatype, int dest, int tag,
             MPI_Comm comm);
int MPI_Isend(const void* buf, int count, MPI_Datatype datatype, int dest, int tag,
              MPI_Comm comm, MPI_Request* request);
int MPI_Issend(const void* buf, int count, MPI_Datatype datatype, int dest, int tag,
               MPI_Comm comm, MPI_Request* request);
int MPI_Recv(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
             MPI_Status* status);
int MPI_Irecv(void* buf, int count, MPI_Datatype datatype, int source, int tag, MPI_Comm comm,
              MPI_Request* request);
int MPI_Probe(int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int* flag, MPI_Status* status);
int MPI_Wait(MPI_Request* request, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request requests[], MPI_Status statuses[]);
int MPI_Test(MPI_Request* request, int* flag, MPI_Status* status);
int MPI_Testall(int count, MPI_Request requests[], int* flag, MPI_Status statuses[]);
int MPI_Get_count(const MPI_Status* status, MPI_Datatype datatype, int* count);

int MPI_Pack(const void* inbuf, int incount, MPI_Datatype datatype, void* outbuf, int outsize,
             int* position, MPI_Comm comm);
int MPI_Unpack(const void* inbuf, int insize, int* position, void* outbuf, int outcount,
               MPI_Datatype datatype, MPI_Comm comm);
int MPI_Pack_size(int incount, MPI_Datatype datatype, MPI_Comm comm, int* size);

/* Not MPI: messages still queued (sent, never received) on any communicator.
 * A correct single-rank run of the reference leaves none. */
int mpi_stub_pending_messages(void);

#ifdef __cplusplus
}
#endif

#endif
