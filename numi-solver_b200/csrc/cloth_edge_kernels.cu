// The frame and batch kernels with the edge/edge yarn self-collision phases
// (solvePrimitiveSelfCollision, applyClothSelfFriction,
// measurePrimitiveSelfPenetration, tools/cloth_bag.cpp:3880-4247), launched
// for schedules with primitiveSelf.  A translation unit of their own, so that
// the default kernels of cloth_api.cu are compiled exactly as without them.
#define NC_EDGE_KERNELS
#include "cloth_frame.cuh"

__global__ void __launch_bounds__(NC_BLOCK_MAX, 1) numi_cloth_frame_edge_kernel(DeviceCloth d, Schedule s) {
    extern __shared__ __align__(16) unsigned char nc_dynamic_smem[];
    run_frame<true, true>(d, s, blockIdx.x, gridDim.x, nc_dynamic_smem);
}

__global__ void __launch_bounds__(NC_BLOCK_MAX, 1) numi_cloth_batch_edge_kernel(const DeviceCloth* cloths, uint32_t count,
                                                                              Schedule s, unsigned int* queue) {
    NC_BATCH_BODY(true)
}
