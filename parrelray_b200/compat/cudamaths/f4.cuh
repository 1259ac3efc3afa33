#pragma once
// The reference splits its vector classes over cudamaths/*.cuh; here they
// all live in vecs.h.
#include "vecs.h"
