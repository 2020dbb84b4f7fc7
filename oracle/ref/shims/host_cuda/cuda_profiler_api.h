// Host-only stand-in (oracle build of the reference): profiler brackets are no-ops.
#pragma once
static inline int cudaProfilerStart() { return 0; }
static inline int cudaProfilerStop() { return 0; }
