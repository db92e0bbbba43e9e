/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_SPMD_H_
#define SHIM_SPMD_H_
#include "shim_chombo.H"
#endif
