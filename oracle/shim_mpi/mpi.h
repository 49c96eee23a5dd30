/* Process-based stand-in for the subset of <mpi.h> that the reference's
 * executables and headers call (test infrastructure and the timed CPU
 * reference arm; nothing in the product links it).
 *
 * MPI_Init forks DSSS_MPI_NP - 1 child processes from the calling process;
 * every rank is a separate process (the reference keeps per-process
 * singletons such as MeasuringTool, so ranks cannot be threads).  Messages
 * travel through shared memory created before the fork: each sender copies
 * a message into its own region of a shared arena and queues a descriptor
 * in the receiver's mailbox; the receiver copies it out.  Sends are buffered
 * (an MPI_Isend completes at once), so no exchange pattern can deadlock on
 * send order.  Collectives are built from these messages on a separate
 * context per communicator, every result reduced in rank order so that all
 * ranks hold identical values.  Matching follows MPI's rules: a message is
 * matched by (communicator, source or MPI_ANY_SOURCE, tag or MPI_ANY_TAG),
 * messages of one sender are not overtaken, and posted receives are served
 * in the order they were posted.
 *
 * Environment: DSSS_MPI_NP (ranks, default 1), DSSS_MPI_ARENA_GB (virtual
 * arena per rank, default 16; pages are only allocated when touched),
 * DSSS_MPI_TIMEOUT (seconds any rank may wait for a message before the job
 * is aborted, default 900).  A rank that dies, aborts or times out takes the
 * whole job down with exit status 2. */
#pragma once
#include <cstdint>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_File;
typedef long long MPI_Aint;
typedef long long MPI_Offset;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
    long long dsss_bytes;
} MPI_Status;

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_REQUEST_NULL 0
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_SEEK_SET 0
#define MPI_MODE_CREATE 1
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_RDWR 8

#define MPI_SUM 1
#define MPI_LAND 2
#define MPI_MAX 3
#define MPI_MIN 4
#define MPI_LOR 5
#define MPI_PROD 6
#define MPI_BAND 7
#define MPI_BOR 8

/* basic types: element size in the low byte, kind in the next */
#define MPI_BYTE 0x001
#define MPI_CHAR 0x101
#define MPI_SHORT 0x202
#define MPI_UNSIGNED_SHORT 0x302
#define MPI_INT 0x404
#define MPI_UNSIGNED 0x504
#define MPI_LONG_LONG_INT 0x608
#define MPI_LONG_LONG 0x608
#define MPI_UNSIGNED_LONG_LONG 0x708
#define MPI_DOUBLE 0x808
#define MPI_LONG 0x908
#define MPI_UNSIGNED_LONG 0xa08
#define MPI_FLOAT 0xb04
#define MPI_UNSIGNED_CHAR 0xc01

extern "C" {
int MPI_Init(int* argc, char*** argv);
int MPI_Initialized(int* flag);
int MPI_Finalize(void);
int MPI_Finalized(int* flag);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Barrier(MPI_Comm comm);

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* newtype);
int MPI_Type_create_struct(int count, const int* blocklens, const MPI_Aint* displs, const MPI_Datatype* types,
                           MPI_Datatype* newtype);
int MPI_Type_get_extent(MPI_Datatype type, MPI_Aint* lb, MPI_Aint* extent);
int MPI_Type_size(MPI_Datatype type, int* size);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);

int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype stype, int dest, int stag, void* rbuf, int rcount,
                 MPI_Datatype rtype, int source, int rtag, MPI_Comm comm, MPI_Status* status);
int MPI_Probe(int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int* flag, MPI_Status* status);
int MPI_Get_count(const MPI_Status* status, MPI_Datatype type, int* count);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* statuses);
int MPI_Test(MPI_Request* req, int* flag, MPI_Status* status);

int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Gather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
               int root, MPI_Comm comm);
int MPI_Gatherv(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, const int* rcounts, const int* displs,
                MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Scatter(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                int root, MPI_Comm comm);
int MPI_Allgather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                  MPI_Comm comm);
int MPI_Allgatherv(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, const int* rcounts,
                   const int* displs, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoall(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                 MPI_Comm comm);
int MPI_Alltoallv(const void* sbuf, const int* scounts, const int* sdispls, MPI_Datatype stype, void* rbuf,
                  const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allreduce(const void* sbuf, void* rbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* sbuf, void* rbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Scan(const void* sbuf, void* rbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Exscan(const void* sbuf, void* rbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);

int MPI_File_open(MPI_Comm comm, const char* name, int amode, MPI_Info info, MPI_File* fh);
int MPI_File_close(MPI_File* fh);
int MPI_File_get_size(MPI_File fh, MPI_Offset* size);
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence);
int MPI_File_read(MPI_File fh, void* buf, int count, MPI_Datatype type, MPI_Status* status);
int MPI_File_write(MPI_File fh, const void* buf, int count, MPI_Datatype type, MPI_Status* status);
}
