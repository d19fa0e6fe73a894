/* Single-rank MPI stand-in used only to compile the reference's CPU path as a
 * test checker (oracle/_ref). Every collective is an identity copy over one
 * rank; point-to-point calls are no-ops because a single rank never has MPI
 * interfaces. Test infrastructure, never linked into the product library. */
#ifndef NDG_ORACLE_STUB_MPI_H
#define NDG_ORACLE_STUB_MPI_H

#include <cstddef>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3

#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_UNSIGNED 4
#define MPI_UNSIGNED_LONG 5
#define MPI_UNSIGNED_LONG_LONG 6
#define MPI_C_BOOL 7

inline std::size_t ndg_stub_mpi_size(MPI_Datatype t) {
    switch (t) {
        case MPI_INT: return sizeof(int);
        case MPI_FLOAT: return sizeof(float);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_UNSIGNED: return sizeof(unsigned);
        case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
        case MPI_UNSIGNED_LONG_LONG: return sizeof(unsigned long long);
        case MPI_C_BOOL: return sizeof(bool);
        default: return 1;
    }
}

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }

inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memmove(recv, send, static_cast<std::size_t>(count) * ndg_stub_mpi_size(t));
    return MPI_SUCCESS;
}

inline int MPI_Allgather(const void* send, int count, MPI_Datatype t, void* recv, int, MPI_Datatype, MPI_Comm) {
    std::memmove(recv, send, static_cast<std::size_t>(count) * ndg_stub_mpi_size(t));
    return MPI_SUCCESS;
}

inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }

inline int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype* t) { *t = 0; return MPI_SUCCESS; }
inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint, MPI_Aint, MPI_Datatype* t) { *t = 0; return MPI_SUCCESS; }
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }

#endif
