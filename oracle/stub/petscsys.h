// Single-process stand-in for the two PETSc/MPI headers that the reference's
// header-only element code includes.  It only defines the scalar typedefs and
// the handful of collective calls those headers touch, with one-rank
// semantics (every reduction is the identity).  Test infrastructure only: it
// lets the oracle build compile the reference element arithmetic unmodified.
#pragma once
#include <cstring>

typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscInt;
typedef int PetscErrorCode;
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

// Datatype handles carry their byte width so the one-rank reduction can copy.
enum { PETSC_COMM_WORLD = 0, PETSC_COMM_SELF = 0, PetscSuccess = 0 };
enum {
	MPI_CHAR = 1, MPI_C_BOOL = 1,
	MPI_INT = 4, MPI_UINT = 4, MPI_UNSIGNED = 4,
	MPI_DOUBLE = 8, MPI_LONG_LONG = 8, MPI_UINT64_T = 8, MPI_UNSIGNED_LONG_LONG = 8, MPI_INT64_T = 8
};
enum { MPI_SUM, MPI_MIN, MPI_MAX, MPI_LOR, MPI_LAND };
#define MPI_IN_PLACE ((void*)1)

inline double PetscRealPart(double value) { return value; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return 0; }
inline int MPI_Allreduce(const void* send, void* receive, int count, MPI_Datatype type, MPI_Op, MPI_Comm)
{
	if (send != MPI_IN_PLACE && send != receive)
		std::memcpy(receive, send, static_cast<std::size_t>(count)*static_cast<std::size_t>(type));
	return 0;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
