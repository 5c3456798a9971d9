/*
 * Entry points of the GPU build of upstream's motion-detection sources (TEST INFRASTRUCTURE
 * ONLY; oracle/Makefile.ref target `ncc`). Upstream's ImageProcessor (image_processor.cpp) and
 * block-match kernels (kernels/block_match_kernels.cu) are compiled unmodified with nvcc and
 * linked against NPP; these two functions restate the host side of upstream's public entry
 * points around them, so that the fixture script can call upstream's own pipeline on a GPU:
 *
 *   ref_motion_detection  <- cuda_toolkit::motion_detection (api/cuda_toolkit.cpp:201-238)
 *   ref_corr_images       <- cuda_toolkit::corr_images      (api/cuda_toolkit.cpp:240-329)
 *
 * Nothing in the product library links or loads this file's library.
 */
#include <vector>

#include "image_processing/image_processor.h"

#define REF_API extern "C" __attribute__((visibility("default")))

static ImageProcessor& processor()
{
    static ImageProcessor p;
    return p;
}

// Each frame is copied into its own pitched device image ([0] = width, the fastest axis), the
// block matcher fills frames x grid float4 vectors (dx, dy, peak, no-shift peak), copied back.
REF_API int ref_motion_detection(const float* images, const NccMotionParameters* params, float* motion_maps)
{
    const uint2 dims = {params->image_dims[0], params->image_dims[1]};
    const size_t pixels = (size_t)dims.x * dims.y;
    std::vector<PitchedArray<float>> d_images;
    d_images.reserve(params->frame_count);
    for (uint i = 0; i < params->frame_count; ++i) {
        float* d = nullptr;
        size_t pitch = 0;
        if (cudaMallocPitch((void**)&d, &pitch, dims.x * sizeof(float), dims.y) != cudaSuccess) return -1;
        if (cudaMemcpy2D(d, pitch, images + i * pixels, dims.x * sizeof(float), dims.x * sizeof(float), dims.y,
                         cudaMemcpyHostToDevice) != cudaSuccess)
            return -1;
        d_images.emplace_back(d, pitch, uint3{dims.x, dims.y, 1});
    }
    cudaDeviceSynchronize();
    const bool ok = processor().ncc_block_match(d_images, reinterpret_cast<float4*>(motion_maps), *params);
    cudaDeviceSynchronize();
    return ok ? 0 : -1;  // the PitchedArray destructors release the images
}

// Valid zero-mean normalised cross-correlation of a template over a source image; dims are
// {width, height}; the map is (ws - wt + 1) x (hs - ht + 1), row-major.
REF_API int ref_corr_images(const float* tpl, const float* src, const unsigned* tpl_dims, const unsigned* src_dims,
                            float* corr)
{
    const uint2 td = {tpl_dims[0], tpl_dims[1]}, sd = {src_dims[0], src_dims[1]};
    if (!td.x || !td.y || !sd.x || !sd.y || td.x > sd.x || td.y > sd.y) return -1;
    float *dt = nullptr, *ds = nullptr;
    size_t pt = 0, ps = 0;
    if (cudaMallocPitch((void**)&dt, &pt, td.x * sizeof(float), td.y) != cudaSuccess) return -1;
    if (cudaMallocPitch((void**)&ds, &ps, sd.x * sizeof(float), sd.y) != cudaSuccess) return -1;
    PitchedArray<float> t(dt, pt, uint3{td.x, td.y, 1}), s(ds, ps, uint3{sd.x, sd.y, 1});
    if (cudaMemcpy2D(dt, pt, tpl, td.x * sizeof(float), td.x * sizeof(float), td.y, cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy2D(ds, ps, src, sd.x * sizeof(float), sd.x * sizeof(float), sd.y, cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return -1;
    return processor().corr_images(t, s, corr, td, sd) ? 0 : -1;
}
