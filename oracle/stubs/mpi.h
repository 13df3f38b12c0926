/* ORACLE test infrastructure: the few MPI declarations the reference's setup sources name, so
 * that its ANM code compiles without an MPI installation.  Nothing on the ANM path calls them
 * (anm_harness.cc defines MPI_Abort to abort the process). */
#pragma once
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
int MPI_Abort(MPI_Comm comm, int code);
