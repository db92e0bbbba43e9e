/* Test infrastructure (oracle reference build): one process, no MPI. */
#ifndef SHIM_MPI_H_
#define SHIM_MPI_H_
inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
#endif
