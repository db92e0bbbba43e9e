/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_REAL_H_
#define SHIM_REAL_H_
#include "shim_chombo.H"
#endif
