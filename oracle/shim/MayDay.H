/* Test infrastructure (oracle reference build): see shim_chombo.H. */
#ifndef SHIM_MAYDAY_H_
#define SHIM_MAYDAY_H_
#include "shim_chombo.H"
#endif
