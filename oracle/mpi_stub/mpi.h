/*
 * Single-rank MPI stand-in used ONLY to compile the unmodified LGF reference
 * sources into the CPU oracle (test infrastructure, never part of the
 * product).  There is no MPI implementation in this image; with one rank
 * every point-to-point loop in the reference is empty
 * (LGF/Field/SU3_field.cpp:366, LGF/Lattice/Lattice.cpp:250), so the only
 * calls that do work are:
 *   - MPI_Allreduce(SUM) on one rank        -> copy
 *   - MPI_File_open/read_at/write_at/close  -> stdio on a FILE*
 * Everything else is a no-op that reports success.
 */
#ifndef LGF_ORACLE_MPI_STUB_H
#define LGF_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef FILE* MPI_File;

#define MPI_SUCCESS 0
#define MPI_ERR_FILE 27
#define MPI_MAX_ERROR_STRING 256
#define MPI_COMM_WORLD 0
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_SUM 0
#define MPI_INFO_NULL 0
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_CREATE 1

static inline int lgf_stub_type_size(MPI_Datatype t) { return t; }

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    memcpy(recv, send, (size_t)count * (size_t)lgf_stub_type_size(t));
    return MPI_SUCCESS;
}

/* never reached with one rank; present so the reference compiles */
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return MPI_SUCCESS; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }

static inline int MPI_Error_class(int code, int* cls) { *cls = code; return MPI_SUCCESS; }
static inline int MPI_Error_string(int code, char* s, int* len) {
    *len = snprintf(s, MPI_MAX_ERROR_STRING, "stub MPI error %d (file could not be opened)", code);
    return MPI_SUCCESS;
}

static inline int MPI_File_open(MPI_Comm, const char* path, int mode, MPI_Info, MPI_File* fh) {
    FILE* f = NULL;
    if (mode & MPI_MODE_RDONLY) {
        f = fopen(path, "rb");
    } else {
        f = fopen(path, "r+b");
        if (!f && (mode & MPI_MODE_CREATE)) f = fopen(path, "w+b");
    }
    *fh = f;
    return f ? MPI_SUCCESS : MPI_ERR_FILE;
}
static inline int MPI_File_close(MPI_File* fh) {
    if (*fh) fclose(*fh);
    *fh = NULL;
    return MPI_SUCCESS;
}
static inline int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char*, MPI_Info) {
    return MPI_SUCCESS;
}
static inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void* buf, int count, MPI_Datatype t, MPI_Status*) {
    if (!fh) return MPI_ERR_FILE;
    if (fseeko(fh, (off_t)off, SEEK_SET) != 0) return MPI_ERR_FILE;
    size_t n = (size_t)count * (size_t)lgf_stub_type_size(t);
    return fread(buf, 1, n, fh) == n ? MPI_SUCCESS : MPI_ERR_FILE;
}
static inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void* buf, int count, MPI_Datatype t, MPI_Status*) {
    if (!fh) return MPI_ERR_FILE;
    if (fseeko(fh, (off_t)off, SEEK_SET) != 0) return MPI_ERR_FILE;
    size_t n = (size_t)count * (size_t)lgf_stub_type_size(t);
    return fwrite(buf, 1, n, fh) == n ? MPI_SUCCESS : MPI_ERR_FILE;
}

#endif
