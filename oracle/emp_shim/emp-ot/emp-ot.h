// emp-ot/emp-ot.h -- TEST INFRASTRUCTURE ONLY.
//
// Stand-in for the reference's umbrella header (ferret/emp-ot/emp-ot/emp-ot.h),
// which pulls in the base-OT protocols and FerretCOT.  The Ferret headers
// compiled from the reference tree (spcot_sender.h, spcot_recver.h, preot.h)
// include it only for emp-tool's names, so it forwards to the emp-tool shim.
#ifndef CUOT_EMP_OT_SHIM_H
#define CUOT_EMP_OT_SHIM_H
#include "emp-tool/emp-tool.h"
#endif
