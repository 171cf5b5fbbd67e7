// Host-only stand-in: thread coordinates are declared in cuda_runtime.h.
#pragma once
#include "cuda_runtime.h"
