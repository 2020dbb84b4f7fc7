// Host-only stand-in (oracle build of the reference): launch parameters live in cuda_runtime.h.
#pragma once
#include "cuda_runtime.h"
