/*
 * MATLAB-facing C entry points. Drop-in for the upstream toolkit's
 * cuda_toolkit/src/public/cuda_toolkit_matlab.h:16-22 (implemented upstream in
 * src/api/cuda_toolkit_matlab.cpp:9-75). The struct is passed by value. The raw
 * size is rf_raw_dim[0]*rf_raw_dim[1] elements and the output is the complex64
 * X*Y*Z volume. Errors are reported on stderr only, as upstream.
 */
#ifndef CUDA_TOOLKIT_MATLAB_H
#define CUDA_TOOLKIT_MATLAB_H

#include "cuda_beamformer_parameters.h"

#if defined(_WIN32)
#define LIB_FN __declspec(dllexport)
#else
#define LIB_FN __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

LIB_FN void beamform_i16_matlab(const short* data, CudaBeamformerParameters bp, float* output);
LIB_FN void beamform_f32_matlab(const float* data, CudaBeamformerParameters bp, float* output);

/* Outside the RF -> volume path: present so the link surface matches; they log and do nothing. */
LIB_FN void motion_detect_f32_matlab(const float* images, NCCMotionParameters params, float* motion_maps);
LIB_FN void corr_images_f32_matlab(const float* template_image, const float* source_image,
                                   CorrImagesParameters params, float* corr_map);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_TOOLKIT_MATLAB_H */
