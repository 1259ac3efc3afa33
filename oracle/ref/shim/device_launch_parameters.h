// Host-only stand-in (oracle build of the reference): everything lives in cuda_runtime.h.
#pragma once
#include "cuda_runtime.h"
