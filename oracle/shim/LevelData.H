/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_LEVELDATA_H_
#define SHIM_LEVELDATA_H_
#include "shim_chombo.H"
#endif
