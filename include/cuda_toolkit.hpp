/*
 * C++ entry point. Drop-in for the upstream toolkit's
 * cuda_toolkit/src/public/cuda_toolkit.hpp:17-29 (implemented upstream in
 * src/api/cuda_toolkit.cpp:109-330).
 *
 * beamform(): input = raw RF bytes (int16 or f32 per bp.data_type, rf_raw_dim[1]
 * channels of rf_raw_dim[0] samples, channel-slowest); output = complex64 volume
 * [Z][Y][X], at least X*Y*Z*8 bytes (checked here; upstream does not check).
 * Synchronous; returns false and logs to stderr on error. Device 0, one call at a
 * time (process-global cached state, like upstream).
 */
#ifndef CUDA_TOOLKIT_HPP
#define CUDA_TOOLKIT_HPP

#ifdef __cplusplus

#if defined(_WIN32)
#define EXPORT_FN __declspec(dllexport)
#else
#define EXPORT_FN __attribute__((visibility("default")))
#endif

#include <cstdint>
#include <span>
#include "cuda_beamformer_parameters.h"

namespace cuda_toolkit
{
    EXPORT_FN bool beamform(std::span<const uint8_t> input_data,
                            std::span<uint8_t> output_data,
                            const CudaBeamformerParameters& bp);

    /* NCC block-matching motion detection over host frames (upstream cuda_toolkit.cpp:202):
     * images holds frame_count float32 frames, motion_maps receives a float4 per grid point and
     * frame (dx, dy, peak, no-shift peak). Returns false and logs on error. */
    EXPORT_FN bool motion_detection(std::span<const uint8_t> images,
                                    std::span<uint8_t> motion_maps,
                                    const NccMotionParameters& params);

    EXPORT_FN bool corr_images(std::span<const float> template_image,
                               std::span<const float> source_image,
                               std::span<float> corr_map,
                               const uint template_dims[2],
                               const uint source_dims[2]);
}

#endif /* __cplusplus */
#endif /* CUDA_TOOLKIT_HPP */
