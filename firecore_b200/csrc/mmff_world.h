// mmff_world.h -- internal view of the device world for the library's other
// translation units (the learned proposal reads systems and parameters from it).
#pragma once
#include <cuda_runtime.h>

#include "mmff_device.cuh"

namespace mmff {

struct WorldView {
    Params P;               // evaluation parameters (no force clamp)
    Systems Y;              // device pointers of the uploaded systems
    cudaStream_t stream;
    int nsys, NA, NV;
    const int4* desc;       // host copy: (aoff, noff, voff, natoms) per system
    double gpos0[3];        // grid origin: world = local + gorg + gpos0
};

// Current systems and parameters; -1 (error message set) when none are uploaded.
int world_view(WorldView* v);
// The world's stream with the device made ready; nullptr (error set) on failure.
cudaStream_t world_stream();

}  // namespace mmff
