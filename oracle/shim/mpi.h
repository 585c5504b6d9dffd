/*
 * Single-rank MPI stand-in used ONLY to compile the reference's own sources
 * into the CPU oracle (test infrastructure; never linked into the product).
 *
 * The reference (src/main.cpp:25, src/class_data.cpp:35-146,
 * src/class_partition.cpp:115-207,1057-1301, src/class_approximation.cpp:171-184,338-352,
 * src/class_approximation-posterior-inference.cpp:235-241,
 * src/class_approximation-predict.cpp:53-95) calls MPI throughout.  With one
 * rank every point-to-point call is unreachable, collectives are copies or
 * no-ops, and MPI-IO maps onto stdio.  Unreachable point-to-point calls abort
 * loudly so that a change in the reference that reaches them cannot go
 * unnoticed.
 */
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Info;
typedef int MPI_Request;
typedef FILE* MPI_File;

struct MPI_Status {
    int count_bytes;
};

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_MODE_RDONLY 1
#define MPI_THREAD_MULTIPLE 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

#define MPI_DOUBLE 8
#define MPI_UNSIGNED_LONG 9
#define MPI_INT 4

static inline int oracle_mpi_type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_DOUBLE: return (int)sizeof(double);
        case MPI_UNSIGNED_LONG: return (int)sizeof(unsigned long);
        case MPI_INT: return (int)sizeof(int);
    }
    std::fprintf(stderr, "oracle mpi shim: unknown datatype %d\n", t);
    std::abort();
}

static inline void oracle_mpi_unreachable(const char* what) {
    std::fprintf(stderr, "oracle mpi shim: %s is unreachable with one rank\n", what);
    std::abort();
}

static inline int MPI_Init_thread(int*, char***, int, int* provided) {
    if (provided) *provided = MPI_THREAD_MULTIPLE;
    return 0;
}
static inline int MPI_Initialized(int* flag) { *flag = 1; return 0; }
static inline int MPI_Finalized(int* flag) { *flag = 1; return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int root, MPI_Comm) {
    if (root != 0) oracle_mpi_unreachable("MPI_Bcast from a non-zero root");
    return 0;
}

static inline int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                                void* recvbuf, int, MPI_Datatype, MPI_Comm) {
    std::memmove(recvbuf, sendbuf, (size_t)sendcount * oracle_mpi_type_size(sendtype));
    return 0;
}

static inline int MPI_Allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                                 void* recvbuf, const int*, const int* displs, MPI_Datatype recvtype,
                                 MPI_Comm) {
    size_t es = (size_t)oracle_mpi_type_size(recvtype);
    std::memmove((char*)recvbuf + (size_t)displs[0] * es, sendbuf,
                 (size_t)sendcount * oracle_mpi_type_size(sendtype));
    return 0;
}

static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
    oracle_mpi_unreachable("MPI_Send");
    return 1;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    oracle_mpi_unreachable("MPI_Recv");
    return 1;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
    oracle_mpi_unreachable("MPI_Isend");
    return 1;
}

static inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 0; return 0; }
static inline int MPI_Group_range_excl(MPI_Group, int, int[][3], MPI_Group*) {
    oracle_mpi_unreachable("MPI_Group_range_excl");
    return 1;
}
static inline int MPI_Comm_create(MPI_Comm, MPI_Group, MPI_Comm*) {
    oracle_mpi_unreachable("MPI_Comm_create");
    return 1;
}

static inline int MPI_File_open(MPI_Comm, const char* name, int, MPI_Info, MPI_File* fh) {
    *fh = std::fopen(name, "rb");
    return *fh ? 0 : 1;
}
static inline int MPI_File_close(MPI_File* fh) {
    if (*fh) std::fclose(*fh);
    *fh = nullptr;
    return 0;
}
static inline int MPI_File_read(MPI_File fh, void* buf, int count, MPI_Datatype type, MPI_Status* st) {
    size_t es = (size_t)oracle_mpi_type_size(type);
    size_t got = fh ? std::fread(buf, es, (size_t)count, fh) : 0;
    if (st) st->count_bytes = (int)(got * es);
    return 0;
}
static inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype type, int* count) {
    *count = st->count_bytes / oracle_mpi_type_size(type);
    return 0;
}
