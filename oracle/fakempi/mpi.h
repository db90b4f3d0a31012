/*
 * Single-rank stand-in for the subset of MPI that the HARM-COOL reference
 * calls.  TEST INFRASTRUCTURE ONLY: it exists so that the reference's own
 * C sources can be compiled into a CPU checker library (oracle/_ref).
 *
 * On one rank the reference relies on MPI for real data movement in two
 * places: the periodic phi halo (self-Sendrecv of whole phi planes,
 * step_ch.c:189-198, flux_ct 3D) and the opposite-phi polar ghosts
 * (bounds.c:161-275).  So Sendrecv/Isend/Irecv here really pack and unpack
 * MPI_Type_create_subarray layouts when the peer is this rank; a peer of
 * MPI_PROC_NULL makes the call a no-op, exactly as MPI specifies.
 */
#ifndef HARM_FAKEMPI_H
#define HARM_FAKEMPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD   ((MPI_Comm)0)
#define MPI_PROC_NULL    (-2)
#define MPI_ANY_SOURCE   (-1)
#define MPI_IN_PLACE     ((void *)1)
#define MPI_INFO_NULL    ((MPI_Info)0)
#define MPI_ORDER_C      0
#define MPI_SUCCESS      0

/* basic datatype handles; derived types get handles >= 16 */
#define MPI_DOUBLE ((MPI_Datatype)1)
#define MPI_INT    ((MPI_Datatype)2)
#define MPI_CHAR   ((MPI_Datatype)3)
#define MPI_BYTE   ((MPI_Datatype)4)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Barrier(MPI_Comm c);
int MPI_Dims_create(int nnodes, int ndims, int dims[]);
int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm c, int rank, int maxdims, int coords[]);
int MPI_Cart_rank(MPI_Comm c, const int coords[], int *rank);
int MPI_Cart_shift(MPI_Comm c, int direction, int disp, int *src, int *dst);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype old,
                             MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rtype, int source, int rtag,
                 MPI_Comm c, MPI_Status *st);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op,
                  MPI_Comm c);
int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm c,
             MPI_Status *st);
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c,
              MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm c,
              MPI_Request *req);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status sts[]);

#ifdef __cplusplus
}
#endif
#endif
