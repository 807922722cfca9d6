/* Minimal stand-in for <mpi.h>: the reference includes it unconditionally
 * (src/spd_k.hpp:3, src/global.cpp:2) but, with MPI compiled out
 * (src/define.hpp:1), only needs the MPI_Comm type. Test infrastructure only. */
#pragma once
typedef int MPI_Comm;
