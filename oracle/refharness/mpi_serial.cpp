// Serial implementations of the MPI entry points declared in mpi.h.
// One rank; every collective is a local copy. Test infrastructure only.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

static void unreachable(const char* what) {
    std::fprintf(stderr, "serial MPI stand-in: %s needs a peer rank, but there is one rank\n", what);
    std::abort();
}

extern "C" {

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm*) { return MPI_SUCCESS; }

int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
    unreachable("MPI_Send");
    return 1;
}
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    unreachable("MPI_Recv");
    return 1;
}
int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype, int, int,
                 MPI_Comm, MPI_Status*) {
    unreachable("MPI_Sendrecv");
    return 1;
}

int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op,
                  MPI_Comm) {
    if (sendbuf != recvbuf) std::memcpy(recvbuf, sendbuf, (size_t)count * (size_t)type);
    return MPI_SUCCESS;
}

int MPI_Scatterv(const void* sendbuf, const int* sendcounts, const int* displs,
                 MPI_Datatype sendtype, void* recvbuf, int, MPI_Datatype, int, MPI_Comm) {
    const char* src = static_cast<const char*>(sendbuf) + (size_t)displs[0] * (size_t)sendtype;
    std::memmove(recvbuf, src, (size_t)sendcounts[0] * (size_t)sendtype);
    return MPI_SUCCESS;
}

int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int,
               MPI_Datatype, int, MPI_Comm) {
    std::memmove(recvbuf, sendbuf, (size_t)sendcount * (size_t)sendtype);
    return MPI_SUCCESS;
}

int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int*, const int* displs, MPI_Datatype recvtype, int, MPI_Comm) {
    char* dst = static_cast<char*>(recvbuf) + (size_t)displs[0] * (size_t)recvtype;
    std::memmove(dst, sendbuf, (size_t)sendcount * (size_t)sendtype);
    return MPI_SUCCESS;
}

int MPI_Type_create_struct(int count, const int* blocklengths, const MPI_Aint* displacements,
                           const MPI_Datatype* types, MPI_Datatype* newtype) {
    long extent = 0;
    for (int i = 0; i < count; ++i) {
        long end = displacements[i] + (long)blocklengths[i] * (long)types[i];
        if (end > extent) extent = end;
    }
    *newtype = (MPI_Datatype)extent;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }

int MPI_Dims_create(int, int ndims, int* dims) {
    for (int i = 0; i < ndims; ++i)
        if (dims[i] == 0) dims[i] = 1;
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int, MPI_Comm* comm_cart) {
    *comm_cart = 1;
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm, int, int, int* source, int* dest) {
    *source = MPI_PROC_NULL;
    *dest = MPI_PROC_NULL;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm, int, int maxdims, int* coords) {
    for (int i = 0; i < maxdims; ++i) coords[i] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_get(MPI_Comm, int maxdims, int* dims, int* periods, int* coords) {
    for (int i = 0; i < maxdims; ++i) {
        dims[i] = 1;
        periods[i] = 0;
        coords[i] = 0;
    }
    return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm, const int*, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}

}  // extern "C"
