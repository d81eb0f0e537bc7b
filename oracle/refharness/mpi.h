/*
 * Single-process stand-in for the MPI library, used only to build the
 * reference solver's own sources into a serial test harness (the oracle's
 * reference build). Test infrastructure: nothing in the product links it.
 *
 * Semantics: one rank (rank 0 of 1). Cartesian shifts return MPI_PROC_NULL,
 * so the reference's halo exchange (Simulation.cpp:270-516) is skipped and
 * no Halo nodes are created (Subdomain.cpp:322-349). Collectives over one
 * rank are copies. Point-to-point calls are never reached with one rank;
 * they abort if they are.
 */
#pragma once
#ifndef ORACLE_SERIAL_MPI_H
#define ORACLE_SERIAL_MPI_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype; /* encodes the byte extent of one element */
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_UNSIGNED ((MPI_Datatype)sizeof(unsigned))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_SUM 1
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

#ifdef __cplusplus
extern "C" {
#endif

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm,
             MPI_Status* status);
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status* status);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Scatterv(const void* sendbuf, const int* sendcounts, const int* displs,
                 MPI_Datatype sendtype, void* recvbuf, int recvcount, MPI_Datatype recvtype,
                 int root, MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
               int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int* recvcounts, const int* displs, MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Type_create_struct(int count, const int* blocklengths, const MPI_Aint* displacements,
                           const MPI_Datatype* types, MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Dims_create(int nnodes, int ndims, int* dims);
int MPI_Cart_create(MPI_Comm old, int ndims, const int* dims, const int* periods, int reorder,
                    MPI_Comm* comm_cart);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int* source, int* dest);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int* coords);
int MPI_Cart_get(MPI_Comm comm, int maxdims, int* dims, int* periods, int* coords);
int MPI_Cart_rank(MPI_Comm comm, const int* coords, int* rank);

#ifdef __cplusplus
}
#endif

#endif
