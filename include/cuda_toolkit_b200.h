/*
 * Device-resident API of the B200 RF -> volume library.
 *
 * The upstream toolkit exposes only host-span entry points (cuda_toolkit::beamform,
 * the MATLAB wrappers) and a GL-buffer front end. Its internal stages are the
 * classes RfProcessor (cuda_toolkit/src/rf_processing/rf_processor.cpp:20-192) and
 * Beamformer (cuda_toolkit/src/beamformer/beamformer.cu:17-197). This header exposes
 * the same stages on caller-owned device memory and a caller-chosen CUDA stream, so
 * they can be timed, captured in a CUDA graph and checked stage by stage:
 *
 *   cutb_decode   <- RfProcessor::convert_decode_strided / convert_strided (rf_processor.cpp:118-173)
 *   cutb_hilbert  <- RfProcessor::hilbert_transform_strided (rf_processor.cpp:175-192)
 *   cutb_das      <- Beamformer::beamform (beamformer.cu:139-197)
 *   cutb_beamform <- the stage sequence of cuda_toolkit::beamform (cuda_toolkit.cpp:153-186)
 *
 * All pointers are plain device pointers; `stream` is a cudaStream_t (NULL = legacy
 * default stream). Calls are asynchronous with respect to the host unless noted.
 * Every function returns false (or NULL / 0) on error, logs one line to stderr
 * (silence with CUTB_LOG=0) and records a code readable with cutb_last_error().
 */
#ifndef CUDA_TOOLKIT_B200_H
#define CUDA_TOOLKIT_B200_H

#include <stddef.h>
#include <stdint.h>
#include "cuda_beamformer_parameters.h"

#if defined(_WIN32)
#define CUTB_API __declspec(dllexport)
#else
#define CUTB_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes returned by cutb_last_error(). */
enum {
    CUTB_OK = 0,
    CUTB_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size or dimension */
    CUTB_ERR_UNSUPPORTED = 2,      /* valid upstream value that this path does not run */
    CUTB_ERR_NOT_INITIALIZED = 3,  /* call order violated (e.g. decode before init) */
    CUTB_ERR_CUDA = 4,             /* a CUDA runtime call failed */
    CUTB_ERR_ALLOCATION = 5,       /* device allocation failed (or injected failure) */
    CUTB_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up */
};

/* Code and message of the most recent failure on the calling thread. */
CUTB_API int cutb_last_error(void);
CUTB_API const char* cutb_last_error_message(void);
CUTB_API void cutb_clear_error(void);

/* Library version, (major << 16) | minor. */
CUTB_API int cutb_version(void);

/* Encoding matrix of order n as generated upstream (hadamard_decoder.cpp:110-222):
 * row-major +1/-1 bytes, ordering HADAMARD (1) or WALSH (2). n = 2^k, 12*2^k or 20*2^k, n <= 1024. */
CUTB_API bool cutb_encoding_matrix(uint n, int ordering, signed char* out);

/* Options that the parameter struct has no field for. Zero-initialise for defaults. */
typedef struct cutb_options {
    int iq_bf16;      /* 1: analytic signal stored as bf16 complex (halves DAS gather bytes) */
    int das_tile;     /* delay-and-sum tile: 0 = chosen from the grid, 1 = 4x8x32, 2 = 8x8x16 (HERCULES and
                         TPW in a y-z plane), 3 = one thread per voxel instead of the staged engine
                         (TPW and UFORCES only; 0 also picks it when the staged windows of a coarse
                         grid would not fit the stage buffers) */
    int decode_tc;    /* 1: int16 decode on int8 tensor cores (hi/lo byte split, exact); needs 32..256
                         transmits in steps of 32 and rows of 8-sample multiples */
    int das_schedule; /* delay-and-sum schedule: 0 = default: one CTA per tile, except that FORCES,
                         TPW and UFORCES split the tiles of a small volume (or of a partial last
                         wave) over several CTAs whose partial sums meet in plan-owned scratch
                         memory; 1 = one CTA per tile; 2 = stream-K when the tiles exceed one wave
                         (the last waves' tiles x stages split evenly over the resident CTAs) */
    int das_rows_per_stage; /* staged delay-and-sum: receive channels per TMA stage, 1..8 (0 = 8);
                               fewer rows mean more stages and block barriers per channel */
    int reserved[11];
} cutb_options;

typedef struct cutb_plan cutb_plan;

/* Validates bp and prepares everything that depends only on it: the decode transform,
 * the channel map, the match-filter spectrum, the delay-and-sum constants and the
 * intermediate device buffers. Synchronous. */
CUTB_API cutb_plan* cutb_plan_create(const CudaBeamformerParameters* bp, const cutb_options* options);
CUTB_API void cutb_plan_destroy(cutb_plan* plan);

/* Byte sizes of the raw input, one analytic-signal buffer [T][C][S] and the output volume [Z][Y][X]. */
CUTB_API size_t cutb_plan_raw_bytes(const cutb_plan* plan);
CUTB_API size_t cutb_plan_iq_bytes(const cutb_plan* plan);
CUTB_API size_t cutb_plan_volume_bytes(const cutb_plan* plan);

/* Convert + reorder + decode: d_raw [R1][R0] (int16 or f32) -> d_out f32 [T][C][S].
 * out_stride 1 writes packed floats; 2 writes complex [T][C][S] with .y = 0. */
CUTB_API bool cutb_decode(cutb_plan* plan, const void* d_raw, size_t raw_bytes, float* d_out, uint out_stride,
                          void* stream);

/* Match-filtered analytic signal of every [T][C] row: d_in f32 with element stride in_stride
 * (1 = packed, 2 = real part of complex) -> d_iq complex [T][C][S] (complex64, or bf16x2
 * when the plan stores bf16). S: any power of two up to 131072, any other count up to 65536
 * (computed as a zero-padded circular convolution of the same result); rows of more than 16384
 * transform points run on a thread-block cluster of 2 to 8 CTAs per row. Longer rows report
 * CUTB_ERR_UNSUPPORTED. */
CUTB_API bool cutb_hilbert(cutb_plan* plan, const float* d_in, uint in_stride, void* d_iq, void* stream);

/* Delay-and-sum of d_iq [T][C][S] into the complex64 volume d_volume [Z][Y][X]. Tiles may be split
 * over several CTAs that combine their partial sums through scratch memory the plan owns (see
 * cutb_options.das_schedule), so calls of one plan must not overlap on the GPU. */
CUTB_API bool cutb_das(cutb_plan* plan, const void* d_iq, void* d_volume, void* stream);

/* Whole pipeline on device memory, intermediates in the plan's own buffers. */
CUTB_API bool cutb_beamform(cutb_plan* plan, const void* d_raw, size_t raw_bytes, void* d_volume, void* stream);

/* Tile shape (x, y, z voxels) of this plan's delay-and-sum; tile id = (tz * ny + ty) * nx + tx
 * with nx = ceil(X / shape[0]) etc. (1, 1, 1) for the one-thread-per-voxel kernel. */
CUTB_API bool cutb_plan_das_tile_shape(const cutb_plan* plan, uint shape[3]);

/* Delay-and-sum of the z-planes z0 .. z1 - 1 of the volume into d_slab [(z1 - z0)][Y][X] (complex64):
 * the tiles of that depth range, unchanged, so slabs of one frame computed on several GPUs and put
 * side by side equal cutb_das of the whole frame. z0 and z1 lie on the tile depth
 * (cutb_plan_das_tile_shape; z1 may also be Z). It serves the sharding of one large frame over
 * several GPUs: every GPU decodes and transforms the whole frame and beamforms its own slab
 * (cuda_ultrasound_toolkit_b200/sharded.py). Staged engine only. No counterpart upstream, whose
 * beamformer runs on one GPU (rf_processor.cpp:47). */
CUTB_API bool cutb_das_zslab(cutb_plan* plan, const void* d_iq, void* d_slab, uint z0, uint z1, void* stream);

/* Delay-and-sum of the listed tiles only (host array of tile ids), each tile's transmit x channel
 * stages split over `splits` CTAs whose partial sums are added atomically, so that a small set of
 * tiles still fills the GPU. d_volume [Z][Y][X] is cleared first; voxels outside the listed tiles
 * stay zero. HERCULES without coherence factor (the factor needs the complete sums). No
 * counterpart upstream: it serves spot checks of a volume against the full delay-and-sum. */
CUTB_API bool cutb_das_tiles(cutb_plan* plan, const void* d_iq, void* d_volume, const int* tiles, uint ntiles,
                             uint splits, void* stream);

/* ---- batched beamforming (no counterpart upstream) --------------------------------------------
 * Many frames of uneven size (each its own parameter block; HERCULES) beamformed together: every
 * frame's decode + Hilbert, then the delay-and-sum: a frame with at least one full wave of tiles
 * (SMs x resident CTAs) gets the single-frame kernel's grid launch; all smaller frames share one
 * persistent launch per kernel variant that takes (frame, tile) work items, heaviest first, from a
 * device counter. The delay-and-sum launches alternate between two internal streams so that one
 * launch's tail overlaps the next. Frames with identical blocks and options share tables; every
 * frame owns its intermediate buffers (allocated here). cutb_batch_das_launches counts the
 * delay-and-sum launches of one run (persistent groups + direct frames).
 * cutb_batch_run: d_raw[i] -> d_volume[i] (complex64 [Z][Y][X]); with use_graph the whole run is
 * captured into a CUDA graph on the first call for a set of pointers and replayed afterwards.
 * Work runs on the batch's own stream, ordered after and before `stream`. */
typedef struct cutb_batch cutb_batch;
CUTB_API cutb_batch* cutb_batch_create(const CudaBeamformerParameters* params, const cutb_options* options,
                                       uint count);
CUTB_API void cutb_batch_destroy(cutb_batch* batch);
CUTB_API bool cutb_batch_run(cutb_batch* batch, const void* const* d_raw, void* const* d_volume, int use_graph,
                             void* stream);
/* cutb_plan_check for every frame's plan. */
CUTB_API bool cutb_batch_check(cutb_batch* batch, void* stream);
CUTB_API int cutb_batch_launches_per_run(const cutb_batch* batch);
CUTB_API int cutb_batch_das_launches(const cutb_batch* batch);

/* Synchronises `stream` and reports whether a kernel of this plan hit a bounded device-side
 * wait (CUTB_ERR_TIMEOUT); clears the flag. cuda_toolkit::beamform calls it on every frame. */
CUTB_API bool cutb_plan_check(cutb_plan* plan, void* stream);

/* Test hook for the bounded waits of the staged delay-and-sum: from the next
 * call on, stage `stage` (transmit x channel-group step, counted from 0 in every CTA) is never
 * issued, so the wait for its copies runs out after wait_limit_cycles (0: the default of about
 * 0.2 s), the CTA stops, waits for the copies it had already issued and leaves; cutb_plan_check
 * then reports CUTB_ERR_TIMEOUT. stage = -1 turns the hook off. The volume of such a call is
 * undefined. No GPU fault is involved: every wait stays bounded. Every sequence runs on the staged
 * engine except TPW / UFORCES plans on the one-thread-per-voxel kernel (das_tile = 3, or 0 on a grid
 * too coarse for the staged windows), which are rejected here. */
CUTB_API bool cutb_debug_das_skip_stage(cutb_plan* plan, int stage, long long wait_limit_cycles);

/* Number of kernels the last cutb_beamform/cutb_decode/cutb_hilbert/cutb_das call launched. */
CUTB_API int cutb_plan_last_launch_count(const cutb_plan* plan);

/* No counterpart in the upstream library. The analytic signal of cutb_hilbert for callers that
 * cannot let a library allocate device memory: applications that own the GPU memory budget (an
 * acquisition loop that reserves its buffers up front, a plugin host that lends its buffers),
 * where cudaMalloc/cudaFree could stall on device-wide synchronisation mid-frame or fail once the
 * host has reserved the memory. No plan and no allocation: d_in holds rows x samples floats with
 * element stride in_stride (1 or 2), d_iq receives rows x samples complex64, taps/ntaps is the
 * match filter in host memory (ntaps <= samples, 0 = none). The FFT tables live in a fixed device
 * array sized for transforms of up to 16384 points (384 KiB, held by every GPU that loads the
 * library until the process exits): rows of up to 16384 samples when the count is a power of two,
 * up to 8192 otherwise. Rows beyond that capacity are rejected with CUTB_ERR_INVALID_ARGUMENT,
 * counts no transform supports with CUTB_ERR_UNSUPPORTED. A call on a stream that is being captured into a
 * CUDA graph is rejected with CUTB_ERR_UNSUPPORTED: the tables are uploaded from host memory that
 * the call frees before a graph could replay the copy. Every call rewrites the array on `stream`;
 * calls that overlap on the GPU race on it and must be serialised. */
CUTB_API bool cutb_hilbert_static(const float* d_in, uint in_stride, void* d_iq, uint samples, size_t rows,
                                  const float* taps, uint ntaps, void* stream);

/* Measures the device's FP32 fused-multiply-add throughput (TFLOP/s) with a short
 * register-only kernel on `stream`; the roofline denominator of the delay-and-sum stage. */
CUTB_API bool cutb_calibrate_fp32(double* tflops, void* stream);

/* Test hook: the next `after` device allocations succeed, then allocations fail until
 * reset with a negative value. Used to exercise the allocation-failure paths. */
CUTB_API void cutb_debug_fail_allocations_after(int after);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_TOOLKIT_B200_H */
