// gpu_tests.h -- stands in for the reference's gpu/gpu_tests.h (debug checks
// that dev_layer.h includes but the Ferret callers never call).
#pragma once
#include "gpu_matrix.h"
