// The frame kernels whose point self contact keeps the reference's
// Gauss-Seidel order (solveSelfCollision, tools/cloth_bag.cpp:4249-4315):
// phase A in parallel, the ordered pass on one CTA where phase A listed
// coupled particles (cloth_frame.cuh).  Launched for cloths created with
// NUMI_CLOTH_SELF_ORDER=reference.  A translation unit of its own, like the
// edge/edge kernels, so that the default kernels are compiled without the
// ordered pass.
#define NC_EDGE_KERNELS
#define NC_SELF_ORDER_KERNELS
#include "cloth_frame.cuh"

__global__ void __launch_bounds__(NC_BLOCK_MAX, 1) numi_cloth_frame_exact_kernel(DeviceCloth d, Schedule s) {
    extern __shared__ __align__(16) unsigned char nc_dynamic_smem[];
    run_frame<false, false>(d, s, blockIdx.x, gridDim.x, nc_dynamic_smem);
}

__global__ void __launch_bounds__(NC_BLOCK_MAX, 1) numi_cloth_frame_edge_exact_kernel(DeviceCloth d, Schedule s) {
    extern __shared__ __align__(16) unsigned char nc_dynamic_smem[];
    run_frame<true, true>(d, s, blockIdx.x, gridDim.x, nc_dynamic_smem);
}
