/* Single-process stand-in for <mpi.h>, used only to compile the reference's
 * header-only distinguishing-prefix code (bloomfilter.hpp, prefix_doubling.hpp)
 * as an oracle cross-check with ONE rank.  With one rank every collective is a
 * local copy; point-to-point calls, which a one-rank run of that code never
 * makes, abort.  Test infrastructure only. */
#pragma once
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_File;
typedef long long MPI_Aint;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_SUCCESS 0
#define MPI_ANY_TAG (-1)
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_SEEK_SET 0
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_SUM 1
#define MPI_LAND 2
#define MPI_MAX 3
#define MPI_MIN 4
#define MPI_LOR 5
#define MPI_BYTE 0x001
#define MPI_CHAR 0x101
#define MPI_SHORT 0x202
#define MPI_UNSIGNED_SHORT 0x302
#define MPI_INT 0x404
#define MPI_UNSIGNED 0x504
#define MPI_LONG_LONG_INT 0x608
#define MPI_UNSIGNED_LONG_LONG 0x708
#define MPI_DOUBLE 0x808
#define MPI_LONG 0x908
#define MPI_UNSIGNED_LONG 0xa08

inline std::vector<long long>& mpi1_types() { static std::vector<long long> t; return t; }
inline long long mpi1_size(MPI_Datatype t) {
    return t < 0x10000 ? (t & 0xff) : mpi1_types()[t - 0x10000];
}
[[noreturn]] inline void mpi1_die(const char* what) {
    std::fprintf(stderr, "single-rank MPI stand-in: %s is not available\n", what);
    std::abort();
}
inline int MPI_Initialized(int* f) { *f = 1; return 0; }
inline int MPI_Finalized(int* f) { *f = 0; return 0; }
inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* nt) {
    mpi1_types().push_back(count * mpi1_size(old));
    *nt = 0x10000 + (int)mpi1_types().size() - 1;
    return 0;
}
inline int MPI_Type_create_struct(int count, const int* bl, const MPI_Aint* disp, const MPI_Datatype* ts, MPI_Datatype* nt) {
    long long ext = 0;
    for (int i = 0; i < count; ++i) {
        long long e = disp[i] + bl[i] * mpi1_size(ts[i]);
        if (e > ext) ext = e;
    }
    mpi1_types().push_back(ext);
    *nt = 0x10000 + (int)mpi1_types().size() - 1;
    return 0;
}
inline int MPI_Type_get_extent(MPI_Datatype t, MPI_Aint* lb, MPI_Aint* ext) { *lb = 0; *ext = mpi1_size(t); return 0; }
inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
inline int MPI_Type_free(MPI_Datatype*) { return 0; }
inline int MPI_Alltoall(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    std::memmove(r, s, (size_t)(sc * mpi1_size(st))); return 0;
}
inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm) {
    long long es = mpi1_size(st);
    std::memmove((char*)r + rd[0] * es, (const char*)s + sd[0] * es, (size_t)(sc[0] * es)); return 0;
}
inline int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    std::memmove(r, s, (size_t)(sc * mpi1_size(st))); return 0;
}
inline int MPI_Allgatherv(const void* s, int sc, MPI_Datatype st, void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm) {
    long long es = mpi1_size(st);
    std::memmove((char*)r + rd[0] * es, s, (size_t)(sc * es)); return 0;
}
inline int MPI_Gather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) {
    std::memmove(r, s, (size_t)(sc * mpi1_size(st))); return 0;
}
inline int MPI_Scatter(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) {
    std::memmove(r, s, (size_t)(sc * mpi1_size(st))); return 0;
}
inline int MPI_Allreduce(const void* s, void* r, int c, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memmove(r, s, (size_t)(c * mpi1_size(t))); return 0;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Scan(const void* s, void* r, int c, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memmove(r, s, (size_t)(c * mpi1_size(t))); return 0;
}
inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { mpi1_die("MPI_Isend"); }
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { mpi1_die("MPI_Irecv"); }
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { mpi1_die("MPI_Send"); }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { mpi1_die("MPI_Recv"); }
inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { mpi1_die("MPI_Sendrecv"); }
inline int MPI_Wait(MPI_Request*, MPI_Status*) { mpi1_die("MPI_Wait"); }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { mpi1_die("MPI_Waitall"); }
inline int MPI_Test(MPI_Request*, int*, MPI_Status*) { mpi1_die("MPI_Test"); }
inline int MPI_File_open(MPI_Comm, const char*, int, MPI_Info, MPI_File*) { mpi1_die("MPI_File_open"); }
inline int MPI_File_close(MPI_File*) { mpi1_die("MPI_File_close"); }
inline int MPI_File_get_size(MPI_File, MPI_Offset*) { mpi1_die("MPI_File_get_size"); }
inline int MPI_File_seek(MPI_File, MPI_Offset, int) { mpi1_die("MPI_File_seek"); }
inline int MPI_File_read(MPI_File, void*, int, MPI_Datatype, MPI_Status*) { mpi1_die("MPI_File_read"); }
inline int MPI_File_write(MPI_File, const void*, int, MPI_Datatype, MPI_Status*) { mpi1_die("MPI_File_write"); }
inline int MPI_Probe(int, int, MPI_Comm, MPI_Status*) { mpi1_die("MPI_Probe"); }
inline int MPI_Get_count(const MPI_Status*, MPI_Datatype, int*) { mpi1_die("MPI_Get_count"); }
