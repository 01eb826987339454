// kern_coll.cu — the device side of the multi-GPU longitudinal wake.
//
// A bunch can be spread over several GPUs (one process each).  The wake kick needs the whole
// bunch's histogram, so between the wake's stages the host all-reduces, over NCCL, the bunch's z
// range and live count and then the bin counts (capi.cpp).  After the first exchange the bin
// geometry and the charge per macroparticle are recomputed here from the global values, with the
// same formulas as the single-GPU setup kernel, so one rank holding the whole bunch gets exactly
// the single-GPU numbers.
#include <cuda_runtime.h>
#include <cstdint>
#include "kernels.h"

namespace accel {

// scr[0] zmin, scr[1] zmax, scr[4] live count (all global after the exchange)
__global__ void k_lw_regeom(double* scr, int nbins, double charge_nc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double mn = scr[0], mx = scr[1], c = scr[4];
    double dz = (mx - mn) / nbins;
    if (!(dz > 0)) dz = 1e-12;
    scr[2] = dz;
    scr[3] = 1.0 / dz;
    scr[5] = (c > 0) ? charge_nc * 1e-9 / c : 0.0;
}

void launch_lw_regeom(double* scr, int nbins, double charge_nc, cudaStream_t s) {
    k_lw_regeom<<<1, 32, 0, s>>>(scr, nbins, charge_nc);
}

}  // namespace accel
