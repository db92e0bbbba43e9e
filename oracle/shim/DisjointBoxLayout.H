/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_DISJOINTBOXLAYOUT_H_
#define SHIM_DISJOINTBOXLAYOUT_H_
#include "shim_chombo.H"
#endif
