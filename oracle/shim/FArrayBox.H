/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_FARRAYBOX_H_
#define SHIM_FARRAYBOX_H_
#include "shim_chombo.H"
#endif
