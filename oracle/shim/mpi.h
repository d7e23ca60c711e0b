// Single-process stand-in for the four MPI calls the reference's
// util/parallelUtil.cpp makes at start-up (rank 0 of 1).
// ORACLE TEST INFRASTRUCTURE ONLY: used to compile the reference's own
// sources here, where no MPI implementation is installed.
#pragma once
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
inline int MPI_Initialized(int *flag) { *flag = 1; return 0; }
inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
