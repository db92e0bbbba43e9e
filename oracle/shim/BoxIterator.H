/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_BOXITERATOR_H_
#define SHIM_BOXITERATOR_H_
#include "shim_chombo.H"
#endif
