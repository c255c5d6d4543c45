/*
 * Single-rank stand-in for the MPI API, used only to compile the reference's CPU code path
 * into the test oracle (oracle/_ref). This is test infrastructure, not product code.
 *
 * One process is rank 0 of a world of size 1. Reductions and gathers copy the send buffer to the
 * receive buffer; point-to-point calls are never reached with one rank and abort if they are.
 */
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype; // encoded as the element size in bytes
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct
{
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_REQUEST_NULL 0

#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_SIGNED_CHAR ((MPI_Datatype)1)
#define MPI_UNSIGNED_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_SHORT ((MPI_Datatype)2)
#define MPI_UNSIGNED_SHORT ((MPI_Datatype)2)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_UNSIGNED ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)4)
#define MPI_LONG ((MPI_Datatype)8)
#define MPI_UNSIGNED_LONG ((MPI_Datatype)8)
#define MPI_LONG_LONG ((MPI_Datatype)8)
#define MPI_LONG_LONG_INT ((MPI_Datatype)8)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)8)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_LONG_DOUBLE ((MPI_Datatype)16)
#define MPI_C_BOOL ((MPI_Datatype)1)
#define MPI_CXX_BOOL ((MPI_Datatype)1)

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_LOR 4
#define MPI_LAND 5

#define MPI_THREAD_MULTIPLE 3
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_FUNNELED 1

inline void oracleMpiUnreachable(const char* what)
{
    std::fprintf(stderr, "single-rank MPI stand-in: %s is not available with one rank\n", what);
    std::abort();
}

inline int oracleMpiCopy(const void* send, void* recv, int count, MPI_Datatype t)
{
    if (send != MPI_IN_PLACE && send != recv && count > 0) { std::memmove(recv, send, size_t(count) * size_t(t)); }
    return MPI_SUCCESS;
}

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Init_thread(int*, char***, int, int* provided)
{
    if (provided) { *provided = MPI_THREAD_MULTIPLE; }
    return MPI_SUCCESS;
}
inline int MPI_Initialized(int* flag)
{
    *flag = 1;
    return MPI_SUCCESS;
}
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r)
{
    *r = 0;
    return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int* s)
{
    *s = 1;
    return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code)
{
    std::exit(code);
    return 0;
}
inline double MPI_Wtime() { return 0.0; }

inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    return oracleMpiCopy(s, r, n, t);
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    return oracleMpiCopy(s, r, n, t);
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm)
{
    return oracleMpiCopy(s, r, n, t);
}
inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* displs, MPI_Datatype,
                          MPI_Comm)
{
    return oracleMpiCopy(s, (char*)r + size_t(displs[0]) * size_t(t), n, t);
}
inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm)
{
    return oracleMpiCopy(s, r, n, t);
}
inline int MPI_Alltoall(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm)
{
    return oracleMpiCopy(s, r, n, t);
}

inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*)
{
    oracleMpiUnreachable("MPI_Isend");
    return 0;
}
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*)
{
    oracleMpiUnreachable("MPI_Irecv");
    return 0;
}
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm)
{
    oracleMpiUnreachable("MPI_Send");
    return 0;
}
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*)
{
    oracleMpiUnreachable("MPI_Recv");
    return 0;
}
inline int MPI_Probe(int, int, MPI_Comm, MPI_Status*)
{
    oracleMpiUnreachable("MPI_Probe");
    return 0;
}
inline int MPI_Get_count(const MPI_Status*, MPI_Datatype, int* c)
{
    *c = 0;
    return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
typedef void(MPI_User_function)(void*, void*, int*, MPI_Datatype*);
inline int MPI_Op_create(MPI_User_function*, int, MPI_Op* op)
{
    *op = MPI_SUM;
    return MPI_SUCCESS;
}
inline int MPI_Op_free(MPI_Op*) { return MPI_SUCCESS; }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
