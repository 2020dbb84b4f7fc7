// ORACLE / TEST INFRASTRUCTURE — never part of the product path.
//
// The reference's own CUDA path built for sm_100a (oracle/_ref/plfbs_ref_gpu):
// Solver_gpu.cu and the kernels it launches, unmodified, compiled as one
// translation unit. LBFS.hpp defines `__constant__ double lattice_weight[15]`
// and both LBFS.cu and Solver_gpu.cu include it: as separate whole-program
// units each would get its own copy, and Solver_gpu.cu's cudaMemcpyToSymbol
// (Solver_gpu.cu:621) would fill a copy the kernels in LBFS.cu never read;
// with relocatable device code the linker rejects the duplicate definition.
// In one unit the header's include guard leaves a single copy. It is the
// reference-kernel timing on the GPU and a second FP64 parity target for the
// library (atomics make it agree to rounding, not bit for bit).
#include "Solver_gpu.cu"
#include "LBFS.cu"
#include "common_kernels.cu"
#include "immersed_boundary_method.cu"
