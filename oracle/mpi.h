/* Test-infrastructure stub: lets the reference's CPU H-matvec
 * (HACApK_MAGMA.c:5-57) compile without MPI.  Single rank only. */
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
