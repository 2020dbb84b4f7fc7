// Host-only stand-in for <cuda.h> (oracle build of the reference): nothing needed.
#pragma once
#include "cuda_runtime.h"
