/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_INTVECT_H_
#define SHIM_INTVECT_H_
#include "shim_chombo.H"
#endif
