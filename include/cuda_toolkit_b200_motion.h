/*
 * Device-resident image correlation and NCC motion detection of the B200 library.
 *
 * Upstream exposes these only as host-span entry points (cuda_toolkit::corr_images and
 * cuda_toolkit::motion_detection, cuda_toolkit.hpp; corr_images_f32_matlab and
 * motion_detect_f32_matlab, cuda_toolkit_matlab.h), which this library also exports with the
 * same semantics. The functions below take caller-owned device memory and a CUDA stream:
 *
 *   cutb_corr_images      <- ImageProcessor::corr_images (image_processing/image_processor.cpp:
 *                            55-128, NPP nppiCrossCorrValid_NormLevel_32f_C1R)
 *   cutb_motion_detection <- ImageProcessor::ncc_block_match (image_processor.cpp:9-52) with
 *                            _compare_images (:130-228) and block_match_pipeline
 *                            (kernels/block_match_kernels.cu:190-241)
 *
 * Images are row-major FP32 with dims[0] = width (the fastest axis) and dims[1] = height. The
 * correlation is the zero-mean normalised cross-correlation at every position where the template
 * lies inside the source; a position where the source window or the template has zero variance
 * yields FLT_MAX, as upstream's NPP call does.
 *
 * Errors: false, one line on stderr, code in cutb_last_error() (cuda_toolkit_b200.h).
 */
#ifndef CUDA_TOOLKIT_B200_MOTION_H
#define CUDA_TOOLKIT_B200_MOTION_H

#include "cuda_toolkit_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* d_corr receives (src_dims[0] - tpl_dims[0] + 1) x (src_dims[1] - tpl_dims[1] + 1) floats,
 * row-major. Scratch comes from the stream-ordered allocator of the current device. */
CUTB_API bool cutb_corr_images(const float* d_template, const float* d_source, const uint tpl_dims[2],
                               const uint src_dims[2], float* d_corr, void* stream);

/* d_frames: params->frame_count images of image_dims[0] x image_dims[1]. d_maps receives
 * frame_count x motion_grid_dims[1] x motion_grid_dims[0] float4 vectors (dx, dy, peak,
 * no-shift peak), zero for the reference frame and for grid points whose patch lies outside the
 * image. One kernel launch (plus a clear of d_maps) for all frames and grid points; each grid
 * point's search window, template and correlation map are held on chip, so windows needing
 * more than 200 KB of shared memory (about 110 x 110 pixels with a 32 x 32 patch) are
 * rejected with CUTB_ERR_UNSUPPORTED. */
CUTB_API bool cutb_motion_detection(const float* d_frames, const NccMotionParameters* params, float* d_maps,
                                    void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_TOOLKIT_B200_MOTION_H */
