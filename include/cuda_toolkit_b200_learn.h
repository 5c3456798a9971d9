/* Project components with no counterpart in the upstream toolkit: the GPU RF simulator and the
 * learned sparse-transmit restoration network (3-D U-Net trained and run by the library's own
 * tcgen05 convolution kernels). Same conventions as cuda_toolkit_b200.h: device pointers,
 * `stream` a cudaStream_t (NULL = legacy default stream), false + cutb_last_error() on failure,
 * no host synchronisation unless stated. */
#ifndef CUDA_TOOLKIT_B200_LEARN_H
#define CUDA_TOOLKIT_B200_LEARN_H

#include "cuda_toolkit_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GPU RF simulator ------------------------------------------------------------------------
 * Row-column array of `array_rows` transmit rows along y and `channels` receive columns along
 * x, both at `pitch`. Transmit event t fires rows t * row_stride + row_offset + k for
 * k < rows_per_transmit (fired together, their echoes add). array_rows = 0 means
 * transmits * row_stride; row_stride = 0 means rows_per_transmit.
 * Echo model: plane-wave transmit along z, receive at the (column, row) crossing point, a
 * 2-cycle Gaussian-windowed tone at the centre frequency per scatterer; Hadamard encoding of
 * the transmit events (encoding 1, Sylvester order `transmits`) or none (0); white Gaussian
 * noise at snr_db (>= 1000: none) from a Philox4x32-10 stream keyed by the frame's seed;
 * scaling to 0.8 * 32767 / max|signal| and rounding to int16. */
typedef struct cutb_sim_config {
    uint transmits;
    uint rows_per_transmit;
    uint channels;
    uint samples;
    float pitch;
    float sampling_frequency;
    float center_frequency;
    float speed_of_sound;
    float snr_db;
    int encoding;
    uint array_rows;
    uint row_stride;
    uint row_offset;
    uint reserved[3];
} cutb_sim_config;

typedef struct cutb_sim cutb_sim;

CUTB_API cutb_sim* cutb_sim_create(const cutb_sim_config* config);
CUTB_API void cutb_sim_destroy(cutb_sim* sim);
/* d_scatterers: `count` float4 (x, y, z, amplitude) in metres; channel_map: host array of
 * `channels` raw channel indices (receive channel c is stored at raw channel map[c]);
 * d_raw: int16 [channels][transmits * samples]; d_gain (optional): the scale applied, so that
 * volume / gain is in the phantom's amplitude units. */
CUTB_API bool cutb_sim_run(cutb_sim* sim, const float* d_scatterers, uint count, const short* channel_map,
                           unsigned long long noise_seed, void* d_raw, float* d_gain, void* stream);
/* Copies the encoded, noisy FP32 frame [transmits][channels][samples] of the last run (before
 * quantisation) to d_dst. */
CUTB_API bool cutb_sim_copy_signal(const cutb_sim* sim, float* d_dst, void* stream);

/* ---- restoration network -----------------------------------------------------------------------
 * Complex64 volumes [n][Z][Y][X]; sides powers of two (16..256, Z up to 1024). Output =
 * in + s * f(in / s), s the per-volume RMS of the input, f the U-Net. */
typedef struct cutb_unet cutb_unet;

CUTB_API cutb_unet* cutb_unet_create(uint X, uint Y, uint Z, uint max_batch, unsigned long long seed);
CUTB_API void cutb_unet_destroy(cutb_unet* net);
CUTB_API size_t cutb_unet_param_count(const cutb_unet* net);        /* trainable (unpadded) */
CUTB_API size_t cutb_unet_param_buffer_size(const cutb_unet* net);  /* floats in the master vector */
CUTB_API uint cutb_unet_layer_count(void);
/* info = {cin, cout, real cin, real cout, level, weight offset, bias offset} (master vector) */
CUTB_API bool cutb_unet_layer_info(const cutb_unet* net, uint layer, unsigned long long info[7]);
CUTB_API bool cutb_unet_get_params(const cutb_unet* net, float* host);        /* synchronises */
CUTB_API bool cutb_unet_set_params(cutb_unet* net, const float* host);        /* synchronises */
CUTB_API bool cutb_unet_get_gradients(const cutb_unet* net, float* host);     /* synchronises */
CUTB_API bool cutb_unet_forward(cutb_unet* net, const void* d_in, void* d_out, uint nvol, void* stream);
/* Loss = sum |in/s + f - target/s|^2 / (nvol * voxels); gradients into the net's buffer. */
CUTB_API bool cutb_unet_compute_gradients(cutb_unet* net, const void* d_in, const void* d_target, uint nvol,
                                          void* stream);
/* compute_gradients followed by one Adam step (beta 0.9 / 0.999). */
CUTB_API bool cutb_unet_train_step(cutb_unet* net, const void* d_in, const void* d_target, uint nvol, float lr,
                                   void* stream);
/* Mean squared normalised residual of the last gradient pass; synchronises; fails with
 * CUTB_ERR_TIMEOUT when a kernel reported a timed-out pipeline wait. */
CUTB_API bool cutb_unet_last_loss(cutb_unet* net, double* mean_sq);
CUTB_API bool cutb_unet_check(cutb_unet* net);

/* Single 3x3x3 convolutions on channel-blocked BF16 volumes [n][c/8][z][y][x][8] (tests/tools).
 * Master weights FP32 [cout][27][cin], tap = (kz * 3 + ky) * 3 + kx. */
CUTB_API bool cutb_conv3d_relayout(const float* d_w, uint cin, uint cout, void* d_wf, void* d_wb, void* stream);
CUTB_API bool cutb_conv3d_forward(const void* d_in, const void* d_wf, const float* d_bias, void* d_out, uint X,
                                  uint Y, uint Z, uint nb, uint cin, uint cout, int relu, int* d_status,
                                  void* stream);
/* Test hook: 1 routes every forward convolution through the per-tap kernel (no halo reuse). */
CUTB_API void cutb_debug_conv3d_force_tap_kernel(int on);
CUTB_API bool cutb_conv3d_weight_grad(const void* d_in, const void* d_dout, float* d_dw, uint X, uint Y, uint Z,
                                      uint nb, uint cin, uint cout, int* d_status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_TOOLKIT_B200_LEARN_H */
