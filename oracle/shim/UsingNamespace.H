/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_USINGNAMESPACE_H_
#define SHIM_USINGNAMESPACE_H_
#include "shim_chombo.H"
#endif
