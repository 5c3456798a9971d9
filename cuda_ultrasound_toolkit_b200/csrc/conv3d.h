// 3x3x3 "same" convolutions on channel-blocked BF16 volumes, computed as implicit GEMMs on
// the 5th-generation tensor cores (tcgen05, FP32 accumulation in TMEM).
//
// Volume layout ("C8"): [n][c / 8][z][y][x][c % 8], BF16 -- eight channels (16 bytes) per
// voxel per channel block. A tensor may be a slice of a wider buffer (a concatenation): it
// then occupies blocks [cb_offset, cb_offset + its blocks) of cb_total blocks per volume.
//
// Weights: the master copy is FP32 [cout][27][cin] with tap = (kz * 3 + ky) * 3 + kx for the
// offsets (kz - 1, ky - 1, kx - 1). The kernels read BF16 relayouts of it:
//   forward       wf[tap][cin / 8][cout][8]          (B operand, K-major)
//   backward-data wb[tap][cout / 8][cin][8] = W[co][26 - tap][ci]   (the transposed, flipped
//                 filter, so that the input gradient is again a forward convolution)
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace cutb {

struct VolumeShape {
    int X, Y, Z, NB;
};

// Epilogue applied to the FP32 accumulators of the forward kernel.
enum ConvEpilogue : int {
    kEpiBias = 0,          // out = acc + bias
    kEpiBiasRelu = 1,      // out = max(acc + bias, 0)
    kEpiMask = 2,          // out = acc * (mask > 0)           (input gradient through a ReLU)
    kEpiComplexOut = 3,    // out_c[v] = res[v] + scale[n] * (acc[0..1] + bias)    (FP32 complex)
    kEpiLossGrad = 4,      // residual MSE loss vs target; out = d loss / d acc     (training)
};

struct ConvFwdArgs {
    VolumeShape shape;
    int cin, cout;                       // channel counts (multiples of 16)
    const __nv_bfloat16* in;             // C8 volume, cin / 8 blocks (the whole buffer)
    const __nv_bfloat16* wf;             // forward weight relayout
    const float* bias;                   // [cout] or null
    __nv_bfloat16* out;                  // C8 output slice
    int out_cb_total, out_cb_offset;
    int epilogue;
    const __nv_bfloat16* mask;           // kEpiMask: C8 slice with the output's shape
    int mask_cb_total, mask_cb_offset;
    const float2* res;                   // kEpiComplexOut / kEpiLossGrad: input volume [n][z][y][x]
    const float* scale;                  // per-volume normalisation s[n]
    float2* out_c;                       // kEpiComplexOut output [n][z][y][x]
    const float2* target;                // kEpiLossGrad target volume
    float* loss;                         // kEpiLossGrad: += sum of squared residuals (normalised)
    float grad_scale;                    // kEpiLossGrad: d loss / d pred = grad_scale * residual
    int* status;                         // device error word (0 = ok)
};

struct ConvWgradArgs {
    VolumeShape shape;
    int cin, cout;
    const __nv_bfloat16* in;             // forward input (C8, cin / 8 blocks)
    const __nv_bfloat16* dout;           // gradient of the forward output (C8, cout / 8 blocks)
    float* dw;                           // += [cout][27][cin] FP32
    int* status;
};

bool conv3d_forward(const ConvFwdArgs& a, cudaStream_t stream);
// Test hook: route every forward convolution through the per-tap kernel.
void conv3d_force_tap_kernel(bool on);
bool conv3d_wgrad(const ConvWgradArgs& a, cudaStream_t stream);

// Helpers on C8 volumes (all BF16 unless noted).
bool c8_avgpool2(const __nv_bfloat16* in, int in_cb_total, int in_cb_offset, int cb, VolumeShape in_shape,
                 __nv_bfloat16* out, cudaStream_t st);
bool c8_upsample2(const __nv_bfloat16* in, int cb, VolumeShape in_shape, __nv_bfloat16* out, int out_cb_total,
                  int out_cb_offset, cudaStream_t st);
// out[v] = skip[v] + (act[v] > 0) * dlow[v / 2] / 8   (input gradient of a 2x average pool
// whose input also feeds a skip connection; skip and act are slices of concat buffers)
bool c8_pool_backward(const __nv_bfloat16* skip, int skip_cb_total, int skip_cb_offset, const __nv_bfloat16* act,
                      int act_cb_total, int act_cb_offset, const __nv_bfloat16* dlow, int cb, VolumeShape high,
                      __nv_bfloat16* out, cudaStream_t st);
// out[u] = sum of the 8 children of u in dhigh (input gradient of a nearest 2x upsample)
bool c8_upsample_backward(const __nv_bfloat16* dhigh, int dhigh_cb_total, int dhigh_cb_offset, int cb,
                          VolumeShape high, __nv_bfloat16* out, cudaStream_t st);
// db[c] += sum over voxels of g (C8, cb blocks)
bool c8_bias_grad(const __nv_bfloat16* g, int cb, VolumeShape shape, float* db, cudaStream_t st);
// Per-volume RMS of a complex volume, then the normalised C8 input (2 real channels of 16).
bool c8_pack_input(const float2* in, VolumeShape shape, float* scale, float* sumsq, __nv_bfloat16* out,
                   cudaStream_t st);

}  // namespace cutb
