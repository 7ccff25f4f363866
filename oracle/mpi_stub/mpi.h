/*
 * Single-rank MPI stand-in used ONLY to compile the reference BioFVM-B sources
 * for the test oracle (oracle/_ref). No MPI implementation is installed in the
 * build image; the reference's LOD solver at one rank only calls MPI_Barrier,
 * and the Isend/Irecv/Wait branches are never taken (rank == size-1 == 0).
 * Every call here is a no-op that reports success, with size 1 / rank 0.
 * Test infrastructure: not part of the product.
 */
#ifndef BFB_ORACLE_MPI_STUB_H
#define BFB_ORACLE_MPI_STUB_H
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Datatype;
typedef int MPI_Info;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_UNSIGNED 3
#define MPI_CHARACTER 4
#define MPI_CHAR 5
#define MPI_INFO_NULL 0
#define MPI_MODE_WRONLY 1
#define MPI_MODE_CREATE 2
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Init_thread(int *, char ***, int req, int *prov) { if (prov) *prov = req; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm, int) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_free(MPI_Comm *) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Cart_create(MPI_Comm, int, int *, int *, int, MPI_Comm *c) { *c = 0; return 0; }
static inline int MPI_Cart_coords(MPI_Comm, int, int n, int *co) { for (int i = 0; i < n; ++i) co[i] = 0; return 0; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) { if (r) *r = 0; return 0; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) { if (r) *r = 0; return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Gather(const void *s, int sc, MPI_Datatype, void *r, int, MPI_Datatype, int, MPI_Comm) { (void)s; (void)sc; (void)r; return 0; }
static inline int MPI_File_open(MPI_Comm, const char *, int, MPI_Info, MPI_File *f) { *f = 0; return 0; }
static inline int MPI_File_close(MPI_File *) { return 0; }
static inline int MPI_File_write(MPI_File, const void *, int, MPI_Datatype, MPI_Status *) { return 0; }
static inline int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char *, MPI_Info) { return 0; }
static inline int MPI_File_set_size(MPI_File, MPI_Offset) { return 0; }
static inline int MPI_File_get_size(MPI_File, MPI_Offset *s) { *s = 0; return 0; }
#endif
