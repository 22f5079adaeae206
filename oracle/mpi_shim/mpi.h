/*
 * Single-rank stand-in for the handful of MPI calls the reference solver makes.
 *
 * TEST INFRASTRUCTURE ONLY: this header lets the unmodified reference sources
 * (Fabian2598/AMG_SchwingerModel, src/*.cpp) compile into the CPU oracle under
 * oracle/_ref/.  Nothing in the product library includes it.
 *
 * Calls used by the reference:
 *   MPI_Init / MPI_Finalize            src/main.cpp:48,176
 *   MPI_Comm_size / MPI_Comm_rank      src/sap.cpp:68-70, src/amg.cpp:5, include/amg.h:106
 *   MPI_Allreduce(DOUBLE_COMPLEX, SUM) src/sap.cpp:113,149
 *   MPI_Barrier                        src/amg.cpp:279,281, src/tests.cpp, src/main.cpp
 *   MPI_Wtime                          include/amg.h:109-111, src/tests.cpp:75-79
 *
 * With one rank an all-reduce of a sum is a copy: each buffer entry has exactly one
 * contributor, so the result is bit-identical to an np = NB/2 run of the reference
 * provided SAPV::sap_blocks_per_proc covers every block of a colour.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <chrono>
#include <complex>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE_COMPLEX 1
#define MPI_DOUBLE 2
#define MPI_INT 3
#define MPI_SUM 0
#define MPI_SUCCESS 0

inline int oracle_mpi_type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_DOUBLE_COMPLEX: return (int)sizeof(std::complex<double>);
        case MPI_DOUBLE: return (int)sizeof(double);
        case MPI_INT: return (int)sizeof(int);
        default: return 1;
    }
}

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

inline int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    if (sendbuf != recvbuf) std::memcpy(recvbuf, sendbuf, (size_t)count * oracle_mpi_type_size(type));
    return MPI_SUCCESS;
}

inline double MPI_Wtime() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

#endif
