// Host-only stand-in: atomicAdd is declared in cuda_runtime.h.
#pragma once
#include "cuda_runtime.h"
