#pragma once
// cudamaths/mat4.cuh of the reference; see mats.h.
#include "mats.h"
