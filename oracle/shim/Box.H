/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_BOX_H_
#define SHIM_BOX_H_
#include "shim_chombo.H"
#endif
