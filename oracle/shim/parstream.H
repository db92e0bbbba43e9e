/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_PARSTREAM_H_
#define SHIM_PARSTREAM_H_
#include "shim_chombo.H"
#endif
