/* One-rank MPI type stub, just enough for the reference's
 * 00_C/PaScaL_TDMA/src/pascal_tdma.hpp to be parsed when its tdmas.cpp
 * (tdma_many, tdma_cycl_many, tdma_single) is compiled as a known-answer
 * oracle.  No MPI routine is declared: tdmas.cpp calls none. */
#ifndef PPF_ORACLE_MPI_STUB_H
#define PPF_ORACLE_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
#endif
