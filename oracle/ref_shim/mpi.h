/*
 * One-rank stand-in for <mpi.h>.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference walk-on-spheres sources include <mpi.h> for their broadcast,
 * reduction and timing calls (src/bvh.cpp:24-109, src/mesh.cpp:272-294,
 * include/wos/runner.hpp:44-263, include/wos/hdf5_io.hpp:39-44).  No MPI is
 * installed here, so this header gives every call used there the meaning it
 * has on a communicator of size one: broadcasts are no-ops, reductions copy
 * the send buffer, the rank is 0 and the size is 1.  Nothing on the
 * walk-on-spheres hot path depends on MPI, so the compiled reference computes
 * exactly what a one-rank `mpirun -np 1 wos ...` computes.
 */
#ifndef WOS_ORACLE_MPI_SHIM_H
#define WOS_ORACLE_MPI_SHIM_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_Op;
typedef ptrdiff_t MPI_Aint;
typedef int MPI_Datatype;   /* builtin types encode their byte size */

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0

#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_LONG_LONG_INT 8
#define MPI_UINT64_T 8

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }

static inline int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm) {
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return 0;
}

static inline size_t wos_shim_type_size(MPI_Datatype type) {
    return type > 0 ? (size_t)type : 0;
}

static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type,
                             MPI_Op op, int root, MPI_Comm comm) {
    (void)op; (void)root; (void)comm;
    if (send != recv) memcpy(recv, send, (size_t)count * wos_shim_type_size(type));
    return 0;
}

static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type,
                                MPI_Op op, MPI_Comm comm) {
    (void)op; (void)comm;
    if (send != recv) memcpy(recv, send, (size_t)count * wos_shim_type_size(type));
    return 0;
}

static inline double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static inline int MPI_Dims_create(int nnodes, int ndims, int *dims) {
    /* size one: every unset extent becomes 1 */
    (void)nnodes;
    for (int i = 0; i < ndims; ++i) {
        if (dims[i] == 0) dims[i] = 1;
    }
    return 0;
}

/* Derived datatypes only describe broadcast layouts; with one rank they are
 * never used to move data. */
static inline int MPI_Get_address(const void *location, MPI_Aint *address) {
    *address = (MPI_Aint)(uintptr_t)location;
    return 0;
}
static inline int MPI_Type_create_struct(int count, const int *lengths, const MPI_Aint *displacements,
                                         const MPI_Datatype *types, MPI_Datatype *out) {
    (void)count; (void)lengths; (void)displacements; (void)types;
    *out = 0;
    return 0;
}
static inline int MPI_Type_create_resized(MPI_Datatype old, MPI_Aint lb, MPI_Aint extent,
                                          MPI_Datatype *out) {
    (void)old; (void)lb;
    *out = (MPI_Datatype)extent;
    return 0;
}
static inline int MPI_Type_commit(MPI_Datatype *type) { (void)type; return 0; }
static inline int MPI_Type_free(MPI_Datatype *type) { (void)type; return 0; }

#endif
