/*
 * Single-rank stand-in for <mpi.h>, used ONLY to compile the reference's own code as a
 * test oracle and CPU baseline: the skip-sequential / sequential scan
 * (tremor/algos/sss/SkipSequential.cpp) and the whole driver with the adaptive planner
 * (tremor_main.cpp, tremor/algos/tremor/*.cpp). MPI is not installed on these machines;
 * with one rank every collective is a local copy, the one-sided template counter is a
 * plain integer, the progress thread never starts (group_size == 1,
 * SkipSequential.cpp:105), and Tremor::searchIndex answers the templates in a plain loop
 * (num_procs == 1, Tremor.cpp:3335) without the point-to-point template distribution,
 * whose calls below therefore stop the process if they are ever reached.
 *
 * Oracle infrastructure: nothing in the product library includes this file.
 */
#ifndef TM_REF_SHIM_MPI_H
#define TM_REF_SHIM_MPI_H

#include <chrono>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Win;
typedef int MPI_Info;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef struct
{
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_WIN_NULL 0
#define MPI_INFO_NULL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_REQUEST_NULL 0
#define MPI_THREAD_MULTIPLE 3
#define MPI_DOUBLE 10
#define MPI_SUM 1
#define MPI_INT 4
#define MPI_FLOAT 5
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_LONG_LONG 9
#define MPI_SUCCESS 0

static inline size_t tm_shim_type_size(MPI_Datatype t)
{
    switch (t)
    {
    case MPI_INT:
    case MPI_FLOAT:
        return 4;
    default:
        return 8;
    }
}

static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm *out) { *out = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline double MPI_Wtime()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static inline int MPI_Iprobe(int, int, MPI_Comm, int *flag, MPI_Status *) { *flag = 0; return 0; }

/* One-sided window: a single local allocation. */
static inline int MPI_Win_allocate(long size, int, MPI_Info, MPI_Comm, void *baseptr, MPI_Win *win)
{
    *(void **)baseptr = std::calloc(1, (size_t)size);
    *win = 1;
    return 0;
}
static inline int MPI_Win_lock_all(int, MPI_Win) { return 0; }
static inline int MPI_Win_unlock_all(MPI_Win) { return 0; }
static inline int MPI_Win_flush(int, MPI_Win) { return 0; }
static inline int MPI_Win_free(MPI_Win *w) { *w = MPI_WIN_NULL; return 0; }
static inline int MPI_Fetch_and_op(const void *, void *, MPI_Datatype, int, long, MPI_Op, MPI_Win)
{
    /* Only reached when group_size > 1, which one rank never is. */
    std::abort();
    return 0;
}

/* Collectives with one rank: root receives its own contribution. */
static inline int MPI_Gather(const void *send, int count, MPI_Datatype t, void *recv, int, MPI_Datatype, int, MPI_Comm)
{
    if (recv && send && count > 0)
        std::memcpy(recv, send, (size_t)count * tm_shim_type_size(t));
    return 0;
}
static inline int MPI_Gatherv(const void *send, int count, MPI_Datatype t, void *recv, const int *, const int *displs,
                              MPI_Datatype, int, MPI_Comm)
{
    if (recv && send && count > 0)
        std::memcpy((char *)recv + (size_t)displs[0] * tm_shim_type_size(t), send, (size_t)count * tm_shim_type_size(t));
    return 0;
}

/* Start-up, communicators and datatypes. */
static inline int MPI_Init_thread(int *, char ***, int required, int *provided)
{
    *provided = required;
    return 0;
}
static inline int MPI_Initialized(int *flag) { *flag = 1; return 0; }
static inline int MPI_Finalized(int *flag) { *flag = 0; return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *out) { *out = c; return 0; }
static inline int MPI_Type_create_struct(int, const int *, const MPI_Aint *, const MPI_Datatype *, MPI_Datatype *t)
{
    *t = 99; /* only ever broadcast to the root itself, which copies nothing */
    return 0;
}
static inline int MPI_Type_commit(MPI_Datatype *) { return 0; }
static inline int MPI_Type_free(MPI_Datatype *t) { *t = 0; return 0; }

/* Collectives with one rank: the root's buffer is the result. */
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Ibcast(void *, int, MPI_Datatype, int, MPI_Comm, MPI_Request *r)
{
    *r = MPI_REQUEST_NULL;
    return 0;
}
static inline int MPI_Allgather(const void *send, int count, MPI_Datatype t, void *recv, int, MPI_Datatype, MPI_Comm)
{
    if (recv && send && count > 0 && recv != send)
        std::memcpy(recv, send, (size_t)count * tm_shim_type_size(t));
    return 0;
}
static inline int MPI_Test(MPI_Request *, int *flag, MPI_Status *) { *flag = 1; return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }

/* Point-to-point messages: only between ranks, so never with one rank. */
static inline int tm_shim_no_peer()
{
    std::abort();
    return 0;
}
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return tm_shim_no_peer(); }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return tm_shim_no_peer(); }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return tm_shim_no_peer(); }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return tm_shim_no_peer(); }

#endif
