/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_PROBLEMDOMAIN_H_
#define SHIM_PROBLEMDOMAIN_H_
#include "shim_chombo.H"
#endif
