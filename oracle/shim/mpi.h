/*
 * Single-rank MPI stand-in used ONLY to compile the reference SEDI sources
 * (stochastic-estimator.cc and its headers) as a CPU oracle on a machine
 * that has no MPI installation.  Test infrastructure, not product code.
 *
 * Every call behaves as MPI does on a one-rank MPI_COMM_WORLD:
 *  - MPI_Comm_size -> 1, MPI_Comm_rank -> 0 (DomainDecomposition.hpp:29-32
 *    then only accepts -p 1x1x1);
 *  - (I)allreduce copies the send buffer into the receive buffer
 *    (DistrAsyncDotProds.hpp:101-110, ValidateSolver.hpp:108-109);
 *  - Wait/Test complete immediately;
 *  - Isend/Irecv are never reached at -p 1x1x1 because every neighbour is
 *    MPI_PROC_NULL (DomainDecomposition.hpp:73-74, CommHalo.hpp:91,102);
 *    they abort loudly if they ever are.
 */
#ifndef SEDI_ORACLE_SHIM_MPI_H
#define SEDI_ORACLE_SHIM_MPI_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0

#define MPI_CHAR 1
#define MPI_FLOAT 4
#define MPI_DOUBLE 8

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

static inline size_t sedi_shim_type_size(MPI_Datatype t) { return (size_t)t; }

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline double MPI_Wtime() {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Abort(MPI_Comm, int code) {
	fflush(stdout);
	fflush(stderr);
	exit(code);
}
static inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
	if (s != r) memcpy(r, s, (size_t)count * sedi_shim_type_size(t));
	return MPI_SUCCESS;
}
static inline int MPI_Iallreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c, MPI_Request *req) {
	*req = MPI_REQUEST_NULL;
	return MPI_Allreduce(s, r, count, t, op, c);
}
static inline int MPI_Wait(MPI_Request *req, MPI_Status *) { *req = MPI_REQUEST_NULL; return MPI_SUCCESS; }
static inline int MPI_Test(MPI_Request *req, int *flag, MPI_Status *) { *req = MPI_REQUEST_NULL; *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
	fprintf(stderr, "single-rank MPI shim: MPI_Isend reached (only -p 1x1x1 is supported)\n");
	abort();
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
	fprintf(stderr, "single-rank MPI shim: MPI_Irecv reached (only -p 1x1x1 is supported)\n");
	abort();
}

#endif
