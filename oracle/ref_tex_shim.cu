// TEST INFRASTRUCTURE: the reference's texture-based DVF inversion
// (nefct/cc/deform/deform_tex.cu.cc:78-168, DeformInvertKernel and its host
// function invert), built unchanged by nvcc from the reference checkout (the
// Makefile extracts the line range into _ref/gen/deform_tex.inc), so the
// library's nefct_warp_invert can be checked against the hardware-filtered
// texture path it replaces.  Only tests load it.
#include <cuda_runtime.h>
#include <string.h>

#include "deform_tex.inc"

extern "C" {

// mx, my, mz: device [nz][ny][nx] displacement components (voxels);
// ix, iy, iz: device outputs of the same shape.  The reference's invert()
// reads the grid from const_image_shape, which its caller
// (deform_invert_tex, :170-181) sets first; so does this wrapper.  Returns
// the CUDA error code (0 = success); invert() synchronises the device.
int ref_tex_invert(const float *mx, const float *my, const float *mz, int nx, int ny, int nz, float *ix, float *iy,
                   float *iz)
{
    const int shape[3] = {nx, ny, nz};
    cudaError_t e = cudaMemcpyToSymbol(const_image_shape, shape, sizeof(shape));
    if (e != cudaSuccess) return (int)e;
    invert(mx, my, mz, nx, ny, nz, ix, iy, iz);
    return (int)cudaGetLastError();
}

}  // extern "C"
