// gpu_matrix.h -- maps the reference's device-matrix header (gpu/gpu_matrix.h,
// included by ferret/emp-ot/emp-ot/ferret/dev_layer.h) onto this library's
// adapter, so that emp-ot's MpcotReg and LpnF2 compile against
// include/cuot_dev_layer.h instead of cuOT's gpu/ library.
#pragma once
#include "cuot_dev_layer.h"
