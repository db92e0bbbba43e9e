/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_VECTOR_H_
#define SHIM_VECTOR_H_
#include "shim_chombo.H"
#endif
