// Single-rank MPI stand-in (TEST INFRASTRUCTURE ONLY); the interface and its
// semantics are described in mpi.h.  Only the reference's parallel sources,
// compiled into oracle/_ref as a checker, link against it.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <deque>
#include <map>
#include <vector>

namespace {

struct Message {
    int tag;
    std::vector<char> data;
};

struct PendingRecv {
    void* buf;
    long long capacity;  // bytes
    int source;
    int tag;
    MPI_Comm comm;
    bool done;
    MPI_Status status;
};

std::map<MPI_Comm, std::deque<Message>> g_queues;
std::map<int, PendingRecv> g_requests;
int g_next_request = 1;
int g_next_comm = 16;
int g_next_group = 16;

long long type_size(MPI_Datatype t) {
    struct DoubleInt { double d; int i; };
    switch (t) {
    case MPI_CHAR: case MPI_BYTE: case MPI_PACKED: return 1;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_LONG: case MPI_LONG_LONG: case MPI_UNSIGNED_LONG: case MPI_DOUBLE: return 8;
    case MPI_DOUBLE_INT: return (long long)sizeof(DoubleInt);
    default:
        std::fprintf(stderr, "mpi stub: unknown datatype %d\n", t);
        std::abort();
    }
}

void check_rank(int r, const char* what) {
    if (r != 0 && r != MPI_ANY_SOURCE) {
        std::fprintf(stderr, "mpi stub: %s names rank %d, but the world has one rank\n", what, r);
        std::abort();
    }
}

void copy_buf(const void* src, void* dst, long long bytes) {
    if (src == MPI_IN_PLACE || src == dst || bytes <= 0) return;
    std::memmove(dst, src, (size_t)bytes);
}

void set_status(MPI_Status* st, int tag, long long bytes) {
    if (!st) return;
    st->MPI_SOURCE = 0;
    st->MPI_TAG = tag;
    st->MPI_ERROR = MPI_SUCCESS;
    st->stub_bytes = bytes;
}

// The oldest queued message on comm that matches (source, tag), or end().
std::deque<Message>::iterator find_message(MPI_Comm comm, int tag) {
    std::deque<Message>& q = g_queues[comm];
    for (auto it = q.begin(); it != q.end(); ++it)
        if (tag == MPI_ANY_TAG || it->tag == tag) return it;
    return q.end();
}

bool try_complete(PendingRecv& r) {
    if (r.done) return true;
    auto it = find_message(r.comm, r.tag);
    if (it == g_queues[r.comm].end()) return false;
    long long n = (long long)it->data.size();
    if (n > r.capacity) n = r.capacity;
    if (n > 0) std::memcpy(r.buf, it->data.data(), (size_t)n);
    set_status(&r.status, it->tag, n);
    g_queues[r.comm].erase(it);
    r.done = true;
    return true;
}

int enqueue(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm) {
    if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
    check_rank(dest, "a send");
    Message m;
    m.tag = tag;
    long long n = (long long)count * type_size(t);
    m.data.resize((size_t)(n > 0 ? n : 0));
    if (n > 0) std::memcpy(m.data.data(), buf, (size_t)n);
    g_queues[comm].push_back(std::move(m));
    return MPI_SUCCESS;
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Initialized(int* flag) { *flag = 1; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { std::exit(code); }

double MPI_Wtime(void) {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }

int MPI_Comm_split(MPI_Comm, int color, int, MPI_Comm* newcomm) {
    *newcomm = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : g_next_comm++;
    return MPI_SUCCESS;
}
int MPI_Comm_dup(MPI_Comm, MPI_Comm* newcomm) { *newcomm = g_next_comm++; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm* comm) {
    g_queues.erase(*comm);
    *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}
int MPI_Comm_group(MPI_Comm, MPI_Group* group) { *group = g_next_group++; return MPI_SUCCESS; }
int MPI_Comm_create_group(MPI_Comm, MPI_Group group, int, MPI_Comm* newcomm) {
    *newcomm = (group == MPI_GROUP_EMPTY) ? MPI_COMM_NULL : g_next_comm++;
    return MPI_SUCCESS;
}
int MPI_Group_incl(MPI_Group, int n, const int ranks[], MPI_Group* newgroup) {
    for (int i = 0; i < n; i++) check_rank(ranks[i], "a group");
    *newgroup = (n == 0) ? MPI_GROUP_EMPTY : g_next_group++;
    return MPI_SUCCESS;
}
int MPI_Group_free(MPI_Group* group) { *group = MPI_GROUP_NULL; return MPI_SUCCESS; }

int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Ibarrier(MPI_Comm, MPI_Request* request) {
    *request = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Bcast(void*, int, MPI_Datatype, int root, MPI_Comm) {
    check_rank(root, "a broadcast");
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op,
                  MPI_Comm) {
    copy_buf(sendbuf, recvbuf, (long long)count * type_size(t));
    return MPI_SUCCESS;
}
int MPI_Iallreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op,
                   MPI_Comm comm, MPI_Request* request) {
    *request = MPI_REQUEST_NULL;
    return MPI_Allreduce(sendbuf, recvbuf, count, t, op, comm);
}
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op, int root,
               MPI_Comm) {
    check_rank(root, "a reduction");
    copy_buf(sendbuf, recvbuf, (long long)count * type_size(t));
    return MPI_SUCCESS;
}
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
               MPI_Datatype, int root, MPI_Comm) {
    check_rank(root, "a gather");
    copy_buf(sendbuf, recvbuf, (long long)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int[], const int displs[], MPI_Datatype recvtype, int root, MPI_Comm) {
    check_rank(root, "a gather");
    copy_buf(sendbuf, (char*)recvbuf + (long long)displs[0] * type_size(recvtype),
             (long long)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
                  MPI_Datatype, MPI_Comm) {
    copy_buf(sendbuf, recvbuf, (long long)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
int MPI_Allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                   const int[], const int displs[], MPI_Datatype recvtype, MPI_Comm) {
    copy_buf(sendbuf, (char*)recvbuf + (long long)displs[0] * type_size(recvtype),
             (long long)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}

int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm) {
    return enqueue(buf, count, t, dest, tag, comm);
}
int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm,
              MPI_Request* request) {
    *request = MPI_REQUEST_NULL;  // buffered at once: nothing left to wait for
    return enqueue(buf, count, t, dest, tag, comm);
}
int MPI_Issend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm,
               MPI_Request* request) {
    return MPI_Isend(buf, count, t, dest, tag, comm, request);
}
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm comm,
              MPI_Request* request) {
    if (source == MPI_PROC_NULL) { *request = MPI_REQUEST_NULL; return MPI_SUCCESS; }
    check_rank(source, "a receive");
    PendingRecv r;
    r.buf = buf;
    r.capacity = (long long)count * type_size(t);
    r.source = source;
    r.tag = tag;
    r.comm = comm;
    r.done = false;
    set_status(&r.status, tag, 0);
    try_complete(r);
    int id = g_next_request++;
    g_requests[id] = r;
    *request = id;
    return MPI_SUCCESS;
}
int MPI_Recv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm comm,
             MPI_Status* status) {
    MPI_Request req;
    MPI_Irecv(buf, count, t, source, tag, comm, &req);
    return MPI_Wait(&req, status);
}
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int* flag, MPI_Status* status) {
    check_rank(source, "a probe");
    auto it = find_message(comm, tag);
    *flag = (it != g_queues[comm].end());
    if (*flag) set_status(status, it->tag, (long long)it->data.size());
    return MPI_SUCCESS;
}
int MPI_Probe(int source, int tag, MPI_Comm comm, MPI_Status* status) {
    int flag = 0;
    MPI_Iprobe(source, tag, comm, &flag, status);
    if (!flag) {
        std::fprintf(stderr, "mpi stub: probe for tag %d on a single rank with no message sent "
                             "(a real MPI would wait forever)\n", tag);
        std::abort();
    }
    return MPI_SUCCESS;
}
int MPI_Test(MPI_Request* request, int* flag, MPI_Status* status) {
    if (*request == MPI_REQUEST_NULL) {
        *flag = 1;
        set_status(status, MPI_ANY_TAG, 0);
        return MPI_SUCCESS;
    }
    auto it = g_requests.find(*request);
    if (it == g_requests.end()) {
        std::fprintf(stderr, "mpi stub: unknown request %d\n", *request);
        std::abort();
    }
    *flag = try_complete(it->second) ? 1 : 0;
    if (*flag) {
        if (status) *status = it->second.status;
        g_requests.erase(it);
        *request = MPI_REQUEST_NULL;
    }
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* request, MPI_Status* status) {
    int flag = 0;
    MPI_Test(request, &flag, status);
    if (!flag) {
        std::fprintf(stderr, "mpi stub: wait on a receive that no send on this single rank "
                             "matches (a real MPI would wait forever)\n");
        std::abort();
    }
    return MPI_SUCCESS;
}
int MPI_Waitall(int count, MPI_Request requests[], MPI_Status statuses[]) {
    for (int i = 0; i < count; i++) MPI_Wait(&requests[i], statuses ? &statuses[i] : MPI_STATUS_IGNORE);
    return MPI_SUCCESS;
}
int MPI_Testall(int count, MPI_Request requests[], int* flag, MPI_Status statuses[]) {
    *flag = 1;
    for (int i = 0; i < count; i++) {
        if (requests[i] == MPI_REQUEST_NULL) continue;
        auto it = g_requests.find(requests[i]);
        if (it == g_requests.end() || !try_complete(it->second)) *flag = 0;
    }
    if (*flag)
        for (int i = 0; i < count; i++)
            MPI_Test(&requests[i], flag, statuses ? &statuses[i] : MPI_STATUS_IGNORE);
    return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status* status, MPI_Datatype t, int* count) {
    long long s = type_size(t);
    *count = (status->stub_bytes % s) ? MPI_UNDEFINED : (int)(status->stub_bytes / s);
    return MPI_SUCCESS;
}

int MPI_Pack(const void* inbuf, int incount, MPI_Datatype t, void* outbuf, int outsize,
             int* position, MPI_Comm) {
    long long n = (long long)incount * type_size(t);
    if (*position + n > outsize) {
        std::fprintf(stderr, "mpi stub: pack overflows its buffer\n");
        std::abort();
    }
    if (n > 0) std::memcpy((char*)outbuf + *position, inbuf, (size_t)n);
    *position += (int)n;
    return MPI_SUCCESS;
}
int MPI_Unpack(const void* inbuf, int insize, int* position, void* outbuf, int outcount,
               MPI_Datatype t, MPI_Comm) {
    long long n = (long long)outcount * type_size(t);
    if (*position + n > insize) {
        std::fprintf(stderr, "mpi stub: unpack reads past its buffer\n");
        std::abort();
    }
    if (n > 0) std::memcpy(outbuf, (const char*)inbuf + *position, (size_t)n);
    *position += (int)n;
    return MPI_SUCCESS;
}
int MPI_Pack_size(int incount, MPI_Datatype t, MPI_Comm, int* size) {
    *size = (int)((long long)incount * type_size(t));
    return MPI_SUCCESS;
}

int mpi_stub_pending_messages(void) {
    int n = 0;
    for (auto& kv : g_queues) n += (int)kv.second.size();
    return n;
}

}  // extern "C"
