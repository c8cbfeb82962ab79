/* Stub of the MPI interface the reference's main.cpp includes -- TEST INFRASTRUCTURE ONLY.
 * Lets oracle/ref_cpu.cpp compile main.cpp (for its CPU acoustic stepper,
 * staggered_grid_extrapolation_2d_pml) without an MPI installation.  Every call is a no-op for a
 * single process of rank 0; nothing here is ever called by the stepper itself. */
#pragma once
typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_SUM 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_IN_PLACE ((void *)1)
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group *g) { *g = 0; return 0; }
static inline int MPI_Group_incl(MPI_Group, int, const int *, MPI_Group *g) { *g = 0; return 0; }
static inline int MPI_Comm_create(MPI_Comm, MPI_Group, MPI_Comm *c) { *c = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Reduce(const void *, void *, int, MPI_Datatype, MPI_Op, int, MPI_Comm) {
  return 0;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  return 0;
}
