/*
 * Buffer-registry C ABI of the RF front end (decode and Hilbert stages).
 *
 * Drop-in for the upstream toolkit's cuda_toolkit/src/public/cuda_toolkit_ogl.h:37-75
 * (implemented upstream in src/api/cuda_toolkit_ogl.cpp:105-273). Same names, same
 * signatures, same bool-plus-stderr error contract. Upstream, the ids handed to
 * register_cuda_buffers are OpenGL shader-storage buffers that CUDA maps on every
 * call. This library runs headless, so an id names a plain device allocation that
 * the caller registered first with cuda_register_device_buffer (the one export
 * that has no upstream counterpart). Everything runs on device 0's legacy default
 * stream and returns after the work is complete, like upstream.
 */
#ifndef CUDA_TOOLKIT_H
#define CUDA_TOOLKIT_H

#include <stddef.h>
#include <stdint.h>

#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifndef MAX_CHANNEL_COUNT
#define MAX_CHANNEL_COUNT 256
#endif

#if defined(_WIN32)
#define EXPORT_FN __declspec(dllexport)
#else
#define EXPORT_FN __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned int uint;
typedef uint16_t u16;
typedef int16_t i16;

/* input_dims = {samples*transmits + padding, raw channels}; decoded_dims = {S, C, T}.
 * Fixes the encoding to Hadamard order, like upstream (cuda_toolkit_ogl.cpp:105-117). */
EXPORT_FN bool init_cuda_configuration(const uint* input_dims, const uint* decoded_dims);

/* rf_data_ssbos: ids of up to 16 complex [T][C][S] buffers; raw_data_ssbo: id of the raw buffer.
 * Every id must have been registered with cuda_register_device_buffer. (upstream :127-160) */
EXPORT_FN bool register_cuda_buffers(const uint* rf_data_ssbos, uint rf_buffer_count, uint raw_data_ssbo);

/* Copies MAX_CHANNEL_COUNT (256) entries; the first C are used. (upstream :162-175) */
EXPORT_FN bool cuda_set_channel_mapping(const i16 channel_mapping[MAX_CHANNEL_COUNT]);

/* Stores the spectrum of the zero-padded taps (no time reversal, i.e. circular
 * convolution with the taps); length 0 disables filtering. Needs init first. (upstream :177-190) */
EXPORT_FN bool cuda_set_match_filter(const float* match_filter, uint length);

/* Reads .x of complex rf buffer input_buffer_idx, writes the analytic signal to output_buffer_idx. (upstream :237-273) */
EXPORT_FN bool cuda_hilbert(uint input_buffer_idx, uint output_buffer_idx);

/* Converts+reorders+decodes int16 raw data at input_offset bytes into the raw buffer;
 * writes complex [T][C][S] with .x = decoded value and .y = 0. (upstream :192-235) */
EXPORT_FN bool cuda_decode(size_t input_offset, uint output_buffer_idx);

/* Frees every device resource of this ABI and forgets all registrations. (upstream :119-125) */
EXPORT_FN void deinit_cuda_configuration(void);

/* No upstream counterpart: stands in for OpenGL buffer registration on a headless
 * machine. Associates id (non-zero) with a caller-owned device allocation of
 * `bytes` bytes on device 0. Re-registering an id replaces it; dptr == NULL removes it. */
EXPORT_FN bool cuda_register_device_buffer(uint id, void* dptr, size_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_TOOLKIT_H */
