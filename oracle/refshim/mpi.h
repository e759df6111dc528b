/* mpi.h -- single-rank stand-in for the MPI API subset the reference sources use.
 * TEST INFRASTRUCTURE ONLY: lets the reference's own FastEddy sources build into
 * oracle/_ref without an MPI installation. One rank; collectives are copies or no-ops;
 * point-to-point calls report an error (they are only reached with more than one rank).
 */
#ifndef FE_REFSHIM_MPI_H
#define FE_REFSHIM_MPI_H
#ifdef __cplusplus
extern "C" {
#endif
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_CHAR 1
#define MPI_CHARACTER 1
#define MPI_INT 2
#define MPI_INTEGER 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Barrier(MPI_Comm c);
double MPI_Wtime(void);
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Wait(MPI_Request *r, MPI_Status *s);
int MPI_Sendrecv(const void *sb, int sc, MPI_Datatype st, int dest, int stag, void *rb, int rc, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm c, MPI_Status *s);
int MPI_Scatter(const void *sb, int sc, MPI_Datatype st, void *rb, int rc, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Gather(const void *sb, int sc, MPI_Datatype st, void *rb, int rc, MPI_Datatype rt, int root, MPI_Comm c);
#ifdef __cplusplus
}
#endif
#endif
