// mpi_stub.cpp -- the one-rank MPI of mpi.h (test infrastructure only).
//
// A datatype is a basic type (its size) or a subarray of a basic type; its
// elements are packed and unpacked in the type map order the MPI standard
// gives a subarray (C order of the subarray; the extent of the type is the
// whole array).  With one rank every collective moves the caller's own
// block from the send side to the receive side, and a message to self is
// packed when it is sent and unpacked into the first matching receive
// (same communicator and tag, in posting order).  Any use a single rank
// cannot satisfy (another rank, a receive that is never matched, sizes that
// differ) aborts with a message.
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>

struct ppf_mpi_type {
    int basic;                 // bytes of a basic type; 0 for a subarray
    int ndims;
    int sizes[8], subsizes[8], starts[8];
    int order;
    MPI_Datatype base;
};

ppf_mpi_type ppf_mpi_double = { 8, 0, {}, {}, {}, 0, nullptr };
ppf_mpi_type ppf_mpi_double_complex = { 16, 0, {}, {}, {}, 0, nullptr };
ppf_mpi_type ppf_mpi_int = { 4, 0, {}, {}, {}, 0, nullptr };

namespace {

[[noreturn]] void die(const char* what)
{
    std::fprintf(stderr, "one-rank MPI: %s\n", what);
    std::abort();
}

long extent(MPI_Datatype t)
{
    if (t->basic) return t->basic;
    long n = 1;
    for (int d = 0; d < t->ndims; ++d) n *= t->sizes[d];
    return n * extent(t->base);
}

long packed_size(MPI_Datatype t)
{
    if (t->basic) return t->basic;
    long n = 1;
    for (int d = 0; d < t->ndims; ++d) n *= t->subsizes[d];
    return n * packed_size(t->base);
}

// walk the elements of `count` items of type t at buf, in type map order
template <typename F>
void walk(char* buf, int count, MPI_Datatype t, F&& f)
{
    const long ext = extent(t);
    for (int c = 0; c < count; ++c) {
        char* item = buf + c * ext;
        if (t->basic) {
            f(item, (long)t->basic);
            continue;
        }
        const int nd = t->ndims;
        // strides of the full array in elements of the base type
        long stride[8];
        long acc = 1;
        for (int q = 0; q < nd; ++q) {
            const int d = (t->order == MPI_ORDER_C) ? nd - 1 - q : q;
            stride[d] = acc;
            acc *= t->sizes[d];
        }
        const long bext = extent(t->base);
        int idx[8] = { 0 };
        long total = 1;
        for (int d = 0; d < nd; ++d) total *= t->subsizes[d];
        for (long e = 0; e < total; ++e) {
            long off = 0;
            for (int d = 0; d < nd; ++d) off += (long)(t->starts[d] + idx[d]) * stride[d];
            walk(item + off * bext, 1, t->base, f);
            // next index, fastest dimension last (C) or first (Fortran)
            for (int q = 0; q < nd; ++q) {
                const int d = (t->order == MPI_ORDER_C) ? nd - 1 - q : q;
                if (++idx[d] < t->subsizes[d]) break;
                idx[d] = 0;
            }
        }
    }
}

std::vector<char> pack(const void* buf, int count, MPI_Datatype t)
{
    std::vector<char> out;
    out.reserve((size_t)(count * packed_size(t)));
    walk(const_cast<char*>(static_cast<const char*>(buf)), count, t,
         [&](char* p, long n) { out.insert(out.end(), p, p + n); });
    return out;
}

void unpack(const std::vector<char>& data, void* buf, int count, MPI_Datatype t)
{
    if ((long)data.size() != count * packed_size(t)) die("message and receive sizes differ");
    size_t pos = 0;
    walk(static_cast<char*>(buf), count, t, [&](char* p, long n) {
        std::memcpy(p, data.data() + pos, (size_t)n);
        pos += (size_t)n;
    });
}

void copy(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
          MPI_Datatype recvtype)
{
    unpack(pack(sendbuf, sendcount, sendtype), recvbuf, recvcount, recvtype);
}

struct Comm {
    int ndims;
    int periods[8];
};
std::vector<Comm> g_comms(1, Comm{ 0, {} });   // [0]: MPI_COMM_WORLD

struct Msg {
    MPI_Comm comm;
    int tag;
    std::vector<char> data;
};
struct Recv {
    bool pending;
    void* buf;
    int count;
    MPI_Datatype type;
    int tag;
    MPI_Comm comm;
};
std::deque<Msg> g_msgs;
std::vector<Recv> g_reqs;

MPI_Request done_request()
{
    g_reqs.push_back(Recv{ false, nullptr, 0, nullptr, 0, 0 });
    return (MPI_Request)(g_reqs.size() - 1);
}

void check_self(int rank)
{
    if (rank != 0) die("a rank other than 0 was addressed");
}

}  // namespace

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code)
{
    std::fprintf(stderr, "one-rank MPI: MPI_Abort(%d)\n", code);
    std::abort();
}
int MPI_Comm_size(MPI_Comm, int* size)
{
    *size = 1;
    return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm, int* rank)
{
    *rank = 0;
    return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
double MPI_Wtime(void)
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int MPI_Cart_create(MPI_Comm, int ndims, const int* dims, const int* periods, int, MPI_Comm* cart)
{
    Comm c{ ndims, {} };
    for (int d = 0; d < ndims; ++d) {
        if (dims[d] != 1) die("a Cartesian grid of more than one rank");
        c.periods[d] = periods[d];
    }
    g_comms.push_back(c);
    *cart = (MPI_Comm)(g_comms.size() - 1);
    return MPI_SUCCESS;
}
int MPI_Cart_sub(MPI_Comm comm, const int* remain, MPI_Comm* sub)
{
    const Comm& p = g_comms.at((size_t)comm);
    Comm c{ 0, {} };
    for (int d = 0; d < p.ndims; ++d)
        if (remain[d]) c.periods[c.ndims++] = p.periods[d];
    g_comms.push_back(c);
    *sub = (MPI_Comm)(g_comms.size() - 1);
    return MPI_SUCCESS;
}
int MPI_Cart_shift(MPI_Comm comm, int direction, int, int* source, int* dest)
{
    const Comm& c = g_comms.at((size_t)comm);
    const bool periodic = direction < c.ndims && c.periods[direction];
    *source = *dest = periodic ? 0 : MPI_PROC_NULL;   // one rank: its own neighbour, or none
    return MPI_SUCCESS;
}
int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm* out)
{
    g_comms.push_back(Comm{ 0, {} });
    *out = (MPI_Comm)(g_comms.size() - 1);
    return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm* comm)
{
    *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int ndims, const int* sizes, const int* subsizes, const int* starts, int order,
                             MPI_Datatype oldtype, MPI_Datatype* newtype)
{
    if (ndims < 1 || ndims > 8) die("subarray rank out of range");
    ppf_mpi_type* t = new ppf_mpi_type{};
    t->basic = 0;
    t->ndims = ndims;
    for (int d = 0; d < ndims; ++d) {
        if (starts[d] < 0 || subsizes[d] < 0 || starts[d] + subsizes[d] > sizes[d]) die("subarray out of bounds");
        t->sizes[d] = sizes[d];
        t->subsizes[d] = subsizes[d];
        t->starts[d] = starts[d];
    }
    t->order = order;
    t->base = oldtype;
    *newtype = t;
    return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype* type)
{
    if (*type && !(*type)->basic) delete *type;
    *type = MPI_DATATYPE_NULL;
    return MPI_SUCCESS;
}

int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req)
{
    *req = done_request();
    if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
    check_self(dest);
    std::vector<char> data = pack(buf, count, type);
    for (Recv& r : g_reqs)
        if (r.pending && r.comm == comm && r.tag == tag) {
            unpack(data, r.buf, r.count, r.type);
            r.pending = false;
            return MPI_SUCCESS;
        }
    g_msgs.push_back(Msg{ comm, tag, std::move(data) });
    return MPI_SUCCESS;
}
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req)
{
    *req = done_request();
    if (source == MPI_PROC_NULL) return MPI_SUCCESS;
    check_self(source);
    for (auto it = g_msgs.begin(); it != g_msgs.end(); ++it)
        if (it->comm == comm && it->tag == tag) {
            unpack(it->data, buf, count, type);
            g_msgs.erase(it);
            return MPI_SUCCESS;
        }
    g_reqs[(size_t)*req] = Recv{ true, buf, count, type, tag, comm };
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* req, MPI_Status*)
{
    if (*req >= 0 && g_reqs.at((size_t)*req).pending) die("a receive was never matched by a send");
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status*)
{
    for (int q = 0; q < n; ++q) MPI_Wait(&reqs[q], MPI_STATUS_IGNORE);
    return MPI_SUCCESS;
}

int MPI_Alltoallw(const void* sendbuf, const int* sendcounts, const int* sdispls, const MPI_Datatype* sendtypes,
                  void* recvbuf, const int* recvcounts, const int* rdispls, const MPI_Datatype* recvtypes, MPI_Comm)
{
    copy(static_cast<const char*>(sendbuf) + sdispls[0], sendcounts[0], sendtypes[0],
         static_cast<char*>(recvbuf) + rdispls[0], recvcounts[0], recvtypes[0]);
    return MPI_SUCCESS;
}
int MPI_Ialltoallw(const void* sendbuf, const int* sendcounts, const int* sdispls, const MPI_Datatype* sendtypes,
                   void* recvbuf, const int* recvcounts, const int* rdispls, const MPI_Datatype* recvtypes,
                   MPI_Comm comm, MPI_Request* req)
{
    *req = done_request();
    return MPI_Alltoallw(sendbuf, sendcounts, sdispls, sendtypes, recvbuf, recvcounts, rdispls, recvtypes, comm);
}
int MPI_Ialltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm, MPI_Request* req)
{
    *req = done_request();
    copy(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
    return MPI_SUCCESS;
}
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
               MPI_Datatype recvtype, int root, MPI_Comm)
{
    check_self(root);
    copy(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
    return MPI_SUCCESS;
}
int MPI_Igather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                MPI_Datatype recvtype, int root, MPI_Comm comm, MPI_Request* req)
{
    *req = done_request();
    return MPI_Gather(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, root, comm);
}
int MPI_Iscatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm, MPI_Request* req)
{
    *req = done_request();
    check_self(root);
    copy(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
    return MPI_SUCCESS;
}
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm)
{
    copy(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, MPI_Comm)
{
    copy(sendbuf, count, type, recvbuf, count, type);   // the reduction of one contribution
    return MPI_SUCCESS;
}
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, int root, MPI_Comm)
{
    check_self(root);
    copy(sendbuf, count, type, recvbuf, count, type);
    return MPI_SUCCESS;
}
