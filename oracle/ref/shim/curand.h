// Host-only stand-in (oracle build of the reference).  The reference's random
// SSAA kernels are never launched by its frame loop (prr.cpp:261-273).
#pragma once
#include "cuda_runtime.h"
