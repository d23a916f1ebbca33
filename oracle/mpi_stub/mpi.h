/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference TIMBIR
 * engine (Source_Code_4D_Fast) on a machine without MPI, as the CPU oracle.
 *
 * Test infrastructure: nothing in the product links this header.
 *
 * With one rank the reference never sends or receives halo slices
 * (Source_Code_4D_Fast/XT_MPI.c:60-79 guard every call on the neighbour rank),
 * and every reduction is a copy of the local value
 * (XT_ICD_update.c:296-312, :651, :900-902; XT_MPI.c:142).
 */
#ifndef XT_ORACLE_MPI_STUB_H
#define XT_ORACLE_MPI_STUB_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_SUM 0
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }

/* The datatype constant is the element size in bytes. */
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c)
{ (void)o; (void)root; (void)c; memmove(r, s, (size_t)n * (size_t)t); return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c)
{ (void)o; (void)c; memmove(r, s, (size_t)n * (size_t)t); return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *q = 0; return 0; }
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *q = 0; return 0; }
static inline int MPI_Wait(MPI_Request *q, MPI_Status *st) { (void)q; (void)st; return 0; }

#endif
