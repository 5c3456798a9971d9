// The sparse-transmit restoration network: a 3-D U-Net that maps a complex volume beamformed
// from a sparse transmit subset to the full-compound volume, trained and run with the
// tensor-core convolutions of conv3d.cu.
//
// Network (4 levels, 3x3x3 "same" convolutions, ReLU, 2x average pooling down, nearest 2x
// upsampling up, skip connections by channel concatenation; ~0.48 M parameters):
//   level 0 (X x Y x Z)   e0a 2->16, e0b 16->16                 d0 32->16, out 16->2
//   level 1 (/2)          e1a 16->32, e1b 32->32                d1 64->16
//   level 2 (/4)          e2a 32->64, e2b 64->64                d2 128->32
//   level 3 (/8)          bottleneck 64->64
// Input: the complex volume divided by its RMS s (2 real channels, padded to 16).
// Output: in + s * f(in / s) -- the network predicts a residual, so a zero last layer is
// the identity and the untrained network returns the sparse volume itself.
// Loss: mean over voxels and volumes of |in / s + f - target / s|^2 (normalised units).
//
// Activations live in C8 buffers; each encoder's second convolution writes straight into
// the first half of the decoder's concatenation buffer at its level, and each upsample
// writes into the second half, so concatenation costs nothing.
//
// Training: forward with the loss epilogue (which also writes the output gradient), then
// the backward chain -- weight gradients (tcgen05, FP32 atomics), input gradients (the
// forward kernel with flipped weights, ReLU masks fused in its epilogue), pooling and
// upsampling gradients, bias gradients -- and one fused Adam + weight-relayout kernel. All
// work is stream-ordered with no host synchronisation, so a step can be captured in a graph.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "common.cuh"
#include "../../include/cuda_toolkit_b200_learn.h"
#include "conv3d.h"

namespace cutb {
namespace {

constexpr int kLayers = 11;
constexpr int kMaxBatchLimit = 64;

struct LayerSpec {
    int cin, cout, cin_real, cout_real, level;
};
// e0a e0b e1a e1b e2a e2b bott d2 d1 d0 out
constexpr LayerSpec kSpecs[kLayers] = {
    {16, 16, 2, 16, 0},  {16, 16, 16, 16, 0}, {16, 32, 16, 32, 1}, {32, 32, 32, 32, 1},
    {32, 64, 32, 64, 2}, {64, 64, 64, 64, 2}, {64, 64, 64, 64, 3}, {128, 32, 128, 32, 2},
    {64, 16, 64, 16, 1}, {32, 16, 32, 16, 0}, {16, 16, 16, 2, 0},
};
enum { E0A, E0B, E1A, E1B, E2A, E2B, BOT, D2, D1, D0, OUT };

struct AdamLayer {
    size_t w_off, b_off;
    int cin, cout;
    __nv_bfloat16* wf;
    __nv_bfloat16* wb;
};
struct AdamTable {
    AdamLayer l[kLayers];
};

// One thread per master parameter: Adam update (when lr > 0) and the BF16 relayouts.
__global__ void adam_relayout_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                                     const float* __restrict__ g, size_t count, const AdamTable tab, float lr,
                                     float b1, float b2, float eps, float c1, float c2)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        float w = p[i];
        if (lr > 0.f) {
            const float gi = g[i];
            const float mi = b1 * m[i] + (1.f - b1) * gi;
            const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
            m[i] = mi;
            v[i] = vi;
            w -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
            p[i] = w;
        }
        int L = 0;
        while (L + 1 < kLayers && i >= tab.l[L + 1].w_off) ++L;
        const AdamLayer& l = tab.l[L];
        if (i >= l.b_off) continue;  // bias: no relayout
        const size_t k = i - l.w_off;
        const int ci = (int)(k % l.cin), tap = (int)((k / l.cin) % 27), co = (int)(k / ((size_t)l.cin * 27));
        const __nv_bfloat16 h = __float2bfloat16_rn(w);
        l.wf[(((size_t)tap * (l.cin / 8) + ci / 8) * l.cout + co) * 8 + (ci & 7)] = h;
        l.wb[(((size_t)(26 - tap) * (l.cout / 8) + co / 8) * l.cin + ci) * 8 + (co & 7)] = h;
    }
}

}  // namespace
}  // namespace cutb

using namespace cutb;

struct cutb_unet {
    int X = 0, Y = 0, Z = 0, max_batch = 0;
    size_t count = 0;  // master parameters (padded layout)
    size_t w_off[kLayers], b_off[kLayers];
    float *p = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    __nv_bfloat16* wbuf = nullptr;  // all wf and wb relayouts
    __nv_bfloat16 *wf[kLayers], *wb[kLayers];
    float *scale = nullptr, *sumsq = nullptr, *loss = nullptr;
    int* status = nullptr;
    long long steps = 0;
    float last_nvol = 0;
    // activations (level-0 plane = X * Y * Z * 16 bytes per block per volume)
    __nv_bfloat16 *x0, *t0, *cat0, *dd0, *gfin, *p1, *t1, *cat1, *dd1, *p2, *t2, *cat2, *dd2, *p3, *bott;
    // gradients
    __nv_bfloat16 *g_dd0, *g_cat0, *g_e0b, *g_t0, *g_dd1, *g_cat1, *g_p1, *g_e1b, *g_t1, *g_dd2, *g_cat2, *g_p2,
        *g_e2b, *g_t2, *g_bott, *g_p3;
    std::vector<void*> allocations;

    VolumeShape level(int l, int nb) const { return {X >> l, Y >> l, Z >> l, nb}; }

    bool alloc(void** ptr, size_t bytes)
    {
        if (device_alloc(ptr, bytes) != cudaSuccess) {
            set_error(CUTB_ERR_ALLOCATION, "U-Net: device allocation of %zu bytes failed.", bytes);
            return false;
        }
        allocations.push_back(*ptr);
        return true;
    }
    bool act(__nv_bfloat16** ptr, int lvl, int blocks)
    {
        const size_t vox = (size_t)(X >> lvl) * (Y >> lvl) * (Z >> lvl);
        return alloc((void**)ptr, vox * 16 * blocks * max_batch);
    }
    ~cutb_unet()
    {
        for (void* a : allocations) device_free(a);
    }

    bool build(unsigned long long seed)
    {
        size_t off = 0, wtotal = 0;
        for (int l = 0; l < kLayers; ++l) {
            w_off[l] = off;
            off += (size_t)kSpecs[l].cout * 27 * kSpecs[l].cin;
            b_off[l] = off;
            off += kSpecs[l].cout;
            wtotal += (size_t)kSpecs[l].cout * 27 * kSpecs[l].cin;
        }
        count = off;
        if (!alloc((void**)&p, count * 4) || !alloc((void**)&m, count * 4) || !alloc((void**)&v, count * 4) ||
            !alloc((void**)&g, count * 4) || !alloc((void**)&wbuf, wtotal * 2 * 2))
            return false;
        size_t woff = 0;
        for (int l = 0; l < kLayers; ++l) {
            const size_t n = (size_t)kSpecs[l].cout * 27 * kSpecs[l].cin;
            wf[l] = wbuf + woff;
            wb[l] = wbuf + woff + n;
            woff += 2 * n;
        }
        if (!alloc((void**)&scale, 4 * max_batch) || !alloc((void**)&sumsq, 4 * max_batch) ||
            !alloc((void**)&loss, 4) || !alloc((void**)&status, 4))
            return false;
        const bool ok = act(&x0, 0, 2) && act(&t0, 0, 2) && act(&cat0, 0, 4) && act(&dd0, 0, 2) && act(&gfin, 0, 2) &&
                        act(&p1, 1, 2) && act(&t1, 1, 4) && act(&cat1, 1, 8) && act(&dd1, 1, 2) && act(&p2, 2, 4) &&
                        act(&t2, 2, 8) && act(&cat2, 2, 16) && act(&dd2, 2, 4) && act(&p3, 3, 8) &&
                        act(&bott, 3, 8) && act(&g_dd0, 0, 2) && act(&g_cat0, 0, 4) && act(&g_e0b, 0, 2) &&
                        act(&g_t0, 0, 2) && act(&g_dd1, 1, 2) && act(&g_cat1, 1, 8) && act(&g_p1, 1, 2) &&
                        act(&g_e1b, 1, 4) && act(&g_t1, 1, 4) && act(&g_dd2, 2, 4) && act(&g_cat2, 2, 16) &&
                        act(&g_p2, 2, 4) && act(&g_e2b, 2, 8) && act(&g_t2, 2, 8) && act(&g_bott, 3, 8) &&
                        act(&g_p3, 3, 8);
        if (!ok) return false;
        CUTB_CUDA_OK(cudaMemset(m, 0, count * 4));
        CUTB_CUDA_OK(cudaMemset(v, 0, count * 4));
        CUTB_CUDA_OK(cudaMemset(g, 0, count * 4));
        CUTB_CUDA_OK(cudaMemset(status, 0, 4));
        CUTB_CUDA_OK(cudaMemset(loss, 0, 4));
        // He-normal initialisation of the real weights (fan-in = 27 * real input channels);
        // padded channels, biases and the last layer start at zero.
        std::vector<float> host(count, 0.f);
        std::mt19937_64 rng(seed);
        for (int l = 0; l < OUT; ++l) {
            const LayerSpec& s = kSpecs[l];
            std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / (27.0 * s.cin_real)));
            for (int co = 0; co < s.cout_real; ++co)
                for (int t = 0; t < 27; ++t)
                    for (int ci = 0; ci < s.cin_real; ++ci)
                        host[w_off[l] + ((size_t)co * 27 + t) * s.cin + ci] = (float)nd(rng);
        }
        return upload(host.data());
    }

    AdamTable table() const
    {
        AdamTable t{};
        for (int l = 0; l < kLayers; ++l) t.l[l] = {w_off[l], b_off[l], kSpecs[l].cin, kSpecs[l].cout, wf[l], wb[l]};
        return t;
    }

    bool update(float lr, cudaStream_t st)
    {
        const float b1 = 0.9f, b2 = 0.999f;
        float c1 = 1.f, c2 = 1.f;
        if (lr > 0.f) {
            ++steps;
            c1 = (float)(1.0 / (1.0 - std::pow(b1, (double)steps)));
            c2 = (float)(1.0 / (1.0 - std::pow(b2, (double)steps)));
        }
        adam_relayout_kernel<<<148 * 4, 256, 0, st>>>(p, m, v, g, count, table(), lr, b1, b2, 1e-8f, c1, c2);
        CUTB_CUDA_OK(cudaGetLastError());
        return true;
    }

    bool upload(const float* host)
    {
        CUTB_CUDA_OK(cudaMemcpy(p, host, count * 4, cudaMemcpyHostToDevice));
        if (!update(0.f, 0)) return false;
        CUTB_CUDA_OK(cudaStreamSynchronize(0));
        return true;
    }

    // One forward convolution of layer l.
    bool conv(int l, int nb, const __nv_bfloat16* in, __nv_bfloat16* out, int out_total, int out_off, int epi,
              cudaStream_t st)
    {
        ConvFwdArgs a{};
        a.shape = level(kSpecs[l].level, nb);
        a.cin = kSpecs[l].cin;
        a.cout = kSpecs[l].cout;
        a.in = in;
        a.wf = wf[l];
        a.bias = p + b_off[l];
        a.out = out;
        a.out_cb_total = out_total;
        a.out_cb_offset = out_off;
        a.epilogue = epi;
        a.status = status;
        return conv3d_forward(a, st);
    }
    // Input gradient of layer l: dx = conv(dz, flipped W), masked by `mask` (null: no mask).
    bool dgrad(int l, int nb, const __nv_bfloat16* dz, __nv_bfloat16* dx, const __nv_bfloat16* mask,
               int mask_total, int mask_off, cudaStream_t st)
    {
        ConvFwdArgs a{};
        a.shape = level(kSpecs[l].level, nb);
        a.cin = kSpecs[l].cout;
        a.cout = kSpecs[l].cin;
        a.in = dz;
        a.wf = wb[l];
        a.out = dx;
        a.out_cb_total = kSpecs[l].cin / 8;
        a.out_cb_offset = 0;
        a.epilogue = mask ? kEpiMask : kEpiBias;
        a.mask = mask;
        a.mask_cb_total = mask_total;
        a.mask_cb_offset = mask_off;
        a.status = status;
        return conv3d_forward(a, st);
    }
    bool wgrad(int l, int nb, const __nv_bfloat16* in, const __nv_bfloat16* dz, cudaStream_t st)
    {
        ConvWgradArgs a{};
        a.shape = level(kSpecs[l].level, nb);
        a.cin = kSpecs[l].cin;
        a.cout = kSpecs[l].cout;
        a.in = in;
        a.dout = dz;
        a.dw = g + w_off[l];
        a.status = status;
        if (!conv3d_wgrad(a, st)) return false;
        return c8_bias_grad(dz, kSpecs[l].cout / 8, a.shape, g + b_off[l], st);
    }

    // Forward through the decoder's last hidden layer (dd0); the output layer is applied by
    // the caller with the epilogue it needs.
    bool body(const float2* in, int nb, cudaStream_t st)
    {
        const VolumeShape s0 = level(0, nb);
        return c8_pack_input(in, s0, scale, sumsq, x0, st) && conv(E0A, nb, x0, t0, 2, 0, kEpiBiasRelu, st) &&
               conv(E0B, nb, t0, cat0, 4, 0, kEpiBiasRelu, st) && c8_avgpool2(cat0, 4, 0, 2, s0, p1, st) &&
               conv(E1A, nb, p1, t1, 4, 0, kEpiBiasRelu, st) && conv(E1B, nb, t1, cat1, 8, 0, kEpiBiasRelu, st) &&
               c8_avgpool2(cat1, 8, 0, 4, level(1, nb), p2, st) && conv(E2A, nb, p2, t2, 8, 0, kEpiBiasRelu, st) &&
               conv(E2B, nb, t2, cat2, 16, 0, kEpiBiasRelu, st) &&
               c8_avgpool2(cat2, 16, 0, 8, level(2, nb), p3, st) && conv(BOT, nb, p3, bott, 8, 0, kEpiBiasRelu, st) &&
               c8_upsample2(bott, 8, level(3, nb), cat2, 16, 8, st) && conv(D2, nb, cat2, dd2, 4, 0, kEpiBiasRelu, st) &&
               c8_upsample2(dd2, 4, level(2, nb), cat1, 8, 4, st) && conv(D1, nb, cat1, dd1, 2, 0, kEpiBiasRelu, st) &&
               c8_upsample2(dd1, 2, level(1, nb), cat0, 4, 2, st) && conv(D0, nb, cat0, dd0, 2, 0, kEpiBiasRelu, st);
    }

    bool forward(const float2* in, float2* out, int nb, cudaStream_t st)
    {
        if (!body(in, nb, st)) return false;
        ConvFwdArgs a{};
        a.shape = level(0, nb);
        a.cin = 16;
        a.cout = 16;
        a.in = dd0;
        a.wf = wf[OUT];
        a.bias = p + b_off[OUT];
        a.epilogue = kEpiComplexOut;
        a.res = in;
        a.scale = scale;
        a.out_c = out;
        a.status = status;
        return conv3d_forward(a, st);
    }

    bool gradients(const float2* in, const float2* target, int nb, cudaStream_t st)
    {
        CUTB_CUDA_OK(cudaMemsetAsync(g, 0, count * 4, st));
        CUTB_CUDA_OK(cudaMemsetAsync(loss, 0, 4, st));
        if (!body(in, nb, st)) return false;
        const VolumeShape s0 = level(0, nb), s1 = level(1, nb), s2 = level(2, nb), s3 = level(3, nb);
        ConvFwdArgs a{};
        a.shape = s0;
        a.cin = 16;
        a.cout = 16;
        a.in = dd0;
        a.wf = wf[OUT];
        a.bias = p + b_off[OUT];
        a.out = gfin;
        a.out_cb_total = 2;
        a.epilogue = kEpiLossGrad;
        a.res = in;
        a.scale = scale;
        a.target = target;
        a.loss = loss;
        a.grad_scale = 2.f / ((float)nb * s0.X * s0.Y * s0.Z);
        a.status = status;
        if (!conv3d_forward(a, st)) return false;
        last_nvol = (float)nb;
        (void)s3;
        return
            // output layer and d0 (level 0)
            wgrad(OUT, nb, dd0, gfin, st) && dgrad(OUT, nb, gfin, g_dd0, dd0, 2, 0, st) &&
            wgrad(D0, nb, cat0, g_dd0, st) && dgrad(D0, nb, g_dd0, g_cat0, cat0, 4, 0, st) &&
            c8_upsample_backward(g_cat0, 4, 2, 2, s0, g_dd1, st) &&
            // d1 (level 1)
            wgrad(D1, nb, cat1, g_dd1, st) && dgrad(D1, nb, g_dd1, g_cat1, cat1, 8, 0, st) &&
            c8_upsample_backward(g_cat1, 8, 4, 4, s1, g_dd2, st) &&
            // d2 (level 2)
            wgrad(D2, nb, cat2, g_dd2, st) && dgrad(D2, nb, g_dd2, g_cat2, cat2, 16, 0, st) &&
            c8_upsample_backward(g_cat2, 16, 8, 8, s2, g_bott, st) &&
            // bottleneck (level 3): its input is a pool output, so no mask
            wgrad(BOT, nb, p3, g_bott, st) && dgrad(BOT, nb, g_bott, g_p3, nullptr, 0, 0, st) &&
            // e2b: skip gradient + pooled gradient through its ReLU
            c8_pool_backward(g_cat2, 16, 0, cat2, 16, 0, g_p3, 8, s2, g_e2b, st) &&
            wgrad(E2B, nb, t2, g_e2b, st) && dgrad(E2B, nb, g_e2b, g_t2, t2, 8, 0, st) &&
            wgrad(E2A, nb, p2, g_t2, st) && dgrad(E2A, nb, g_t2, g_p2, nullptr, 0, 0, st) &&
            c8_pool_backward(g_cat1, 8, 0, cat1, 8, 0, g_p2, 4, s1, g_e1b, st) &&
            wgrad(E1B, nb, t1, g_e1b, st) && dgrad(E1B, nb, g_e1b, g_t1, t1, 4, 0, st) &&
            wgrad(E1A, nb, p1, g_t1, st) && dgrad(E1A, nb, g_t1, g_p1, nullptr, 0, 0, st) &&
            c8_pool_backward(g_cat0, 4, 0, cat0, 4, 0, g_p1, 2, s0, g_e0b, st) &&
            wgrad(E0B, nb, t0, g_e0b, st) && dgrad(E0B, nb, g_e0b, g_t0, t0, 2, 0, st) &&
            wgrad(E0A, nb, x0, g_t0, st);
    }
};

namespace {
bool check_net(const cutb_unet* net, unsigned nvol)
{
    CUTB_REQUIRE(net, CUTB_ERR_INVALID_ARGUMENT, "Null U-Net.");
    CUTB_REQUIRE(nvol >= 1 && (int)nvol <= net->max_batch, CUTB_ERR_INVALID_ARGUMENT,
                 "Volume count %u outside 1..%d.", nvol, net->max_batch);
    return true;
}
}  // namespace

extern "C" {

CUTB_API cutb_unet* cutb_unet_create(unsigned X, unsigned Y, unsigned Z, unsigned max_batch, unsigned long long seed)
{
    if (!(is_pow2(X) && is_pow2(Y) && is_pow2(Z) && X >= 16 && Y >= 16 && Z >= 16 && X <= 256 && Y <= 256 &&
          Z <= 1024)) {
        set_error(CUTB_ERR_UNSUPPORTED, "U-Net volume %u x %u x %u: sides must be powers of two, 16..256 (z: 1024).",
                  X, Y, Z);
        return nullptr;
    }
    if (max_batch < 1 || max_batch > (unsigned)kMaxBatchLimit) {
        set_error(CUTB_ERR_INVALID_ARGUMENT, "U-Net batch %u outside 1..%d.", max_batch, kMaxBatchLimit);
        return nullptr;
    }
    auto* net = new cutb_unet();
    net->X = (int)X;
    net->Y = (int)Y;
    net->Z = (int)Z;
    net->max_batch = (int)max_batch;
    if (!net->build(seed)) {
        delete net;
        return nullptr;
    }
    return net;
}

CUTB_API void cutb_unet_destroy(cutb_unet* net)
{
    if (net) cudaDeviceSynchronize();
    delete net;
}

CUTB_API size_t cutb_unet_param_buffer_size(const cutb_unet* net) { return net ? net->count : 0; }

CUTB_API size_t cutb_unet_param_count(const cutb_unet* net)
{
    (void)net;
    size_t n = 0;
    for (int l = 0; l < kLayers; ++l) n += (size_t)kSpecs[l].cout_real * (27 * kSpecs[l].cin_real + 1);
    return n;
}

CUTB_API unsigned cutb_unet_layer_count(void) { return kLayers; }

// info = {cin, cout, cin_real, cout_real, level, weight offset, bias offset}
CUTB_API bool cutb_unet_layer_info(const cutb_unet* net, unsigned layer, unsigned long long info[7])
{
    CUTB_REQUIRE(net && info && layer < (unsigned)kLayers, CUTB_ERR_INVALID_ARGUMENT, "Bad layer query.");
    const LayerSpec& s = kSpecs[layer];
    const unsigned long long v[7] = {(unsigned)s.cin,   (unsigned)s.cout,     (unsigned)s.cin_real, (unsigned)s.cout_real,
                                     (unsigned)s.level, net->w_off[layer], net->b_off[layer]};
    std::memcpy(info, v, sizeof(v));
    return true;
}

CUTB_API bool cutb_unet_get_params(const cutb_unet* net, float* host)
{
    CUTB_REQUIRE(net && host, CUTB_ERR_INVALID_ARGUMENT, "Null argument.");
    CUTB_CUDA_OK(cudaDeviceSynchronize());
    CUTB_CUDA_OK(cudaMemcpy(host, net->p, net->count * 4, cudaMemcpyDeviceToHost));
    return true;
}

CUTB_API bool cutb_unet_set_params(cutb_unet* net, const float* host)
{
    CUTB_REQUIRE(net && host, CUTB_ERR_INVALID_ARGUMENT, "Null argument.");
    CUTB_CUDA_OK(cudaDeviceSynchronize());
    return net->upload(host);
}

CUTB_API bool cutb_unet_get_gradients(const cutb_unet* net, float* host)
{
    CUTB_REQUIRE(net && host, CUTB_ERR_INVALID_ARGUMENT, "Null argument.");
    CUTB_CUDA_OK(cudaDeviceSynchronize());
    CUTB_CUDA_OK(cudaMemcpy(host, net->g, net->count * 4, cudaMemcpyDeviceToHost));
    return true;
}

CUTB_API bool cutb_unet_forward(cutb_unet* net, const void* d_in, void* d_out, unsigned nvol, void* stream)
{
    if (!check_net(net, nvol)) return false;
    CUTB_REQUIRE(d_in && d_out, CUTB_ERR_INVALID_ARGUMENT, "Null volume.");
    return net->forward((const float2*)d_in, (float2*)d_out, (int)nvol, (cudaStream_t)stream);
}

CUTB_API bool cutb_unet_compute_gradients(cutb_unet* net, const void* d_in, const void* d_target, unsigned nvol,
                                          void* stream)
{
    if (!check_net(net, nvol)) return false;
    CUTB_REQUIRE(d_in && d_target, CUTB_ERR_INVALID_ARGUMENT, "Null volume.");
    return net->gradients((const float2*)d_in, (const float2*)d_target, (int)nvol, (cudaStream_t)stream);
}

CUTB_API bool cutb_unet_train_step(cutb_unet* net, const void* d_in, const void* d_target, unsigned nvol, float lr,
                                   void* stream)
{
    if (!check_net(net, nvol)) return false;
    CUTB_REQUIRE(d_in && d_target, CUTB_ERR_INVALID_ARGUMENT, "Null volume.");
    CUTB_REQUIRE(lr > 0.f && std::isfinite(lr), CUTB_ERR_INVALID_ARGUMENT, "Learning rate must be positive.");
    cudaStream_t st = (cudaStream_t)stream;
    return net->gradients((const float2*)d_in, (const float2*)d_target, (int)nvol, st) && net->update(lr, st);
}

// Mean squared residual (normalised units, per real component) of the last gradient pass and
// the device status word; synchronises the device.
CUTB_API bool cutb_unet_last_loss(cutb_unet* net, double* mean_sq)
{
    CUTB_REQUIRE(net && mean_sq, CUTB_ERR_INVALID_ARGUMENT, "Null argument.");
    CUTB_CUDA_OK(cudaDeviceSynchronize());
    float l = 0.f;
    int s = 0;
    CUTB_CUDA_OK(cudaMemcpy(&l, net->loss, 4, cudaMemcpyDeviceToHost));
    CUTB_CUDA_OK(cudaMemcpy(&s, net->status, 4, cudaMemcpyDeviceToHost));
    CUTB_REQUIRE(s == 0, CUTB_ERR_TIMEOUT, "U-Net kernels reported status 0x%x (a pipeline wait timed out).", s);
    const double n = (double)net->last_nvol * net->X * net->Y * net->Z * 2.0;
    *mean_sq = n > 0 ? (double)l / n : 0.0;
    return true;
}

CUTB_API bool cutb_unet_check(cutb_unet* net)
{
    CUTB_REQUIRE(net, CUTB_ERR_INVALID_ARGUMENT, "Null U-Net.");
    CUTB_CUDA_OK(cudaDeviceSynchronize());
    int s = 0;
    CUTB_CUDA_OK(cudaMemcpy(&s, net->status, 4, cudaMemcpyDeviceToHost));
    CUTB_REQUIRE(s == 0, CUTB_ERR_TIMEOUT, "U-Net kernels reported status 0x%x (a pipeline wait timed out).", s);
    return true;
}

// ---- single convolutions (tests and tools) ---------------------------------------------------
CUTB_API void cutb_debug_conv3d_force_tap_kernel(int on) { conv3d_force_tap_kernel(on != 0); }

CUTB_API bool cutb_conv3d_relayout(const float* d_w, unsigned cin, unsigned cout, void* d_wf, void* d_wb, void* stream)
{
    CUTB_REQUIRE(d_w && d_wf && d_wb && cin % 16 == 0 && cout % 16 == 0 && cin && cout, CUTB_ERR_INVALID_ARGUMENT,
                 "conv3d relayout: bad arguments.");
    AdamTable t{};
    const size_t n = (size_t)cout * 27 * cin;
    for (int l = 0; l < kLayers; ++l) t.l[l] = {n + 1, n + 1, (int)cin, (int)cout, nullptr, nullptr};
    t.l[0] = {0, n, (int)cin, (int)cout, (__nv_bfloat16*)d_wf, (__nv_bfloat16*)d_wb};
    adam_relayout_kernel<<<148 * 4, 256, 0, (cudaStream_t)stream>>>(const_cast<float*>(d_w), nullptr, nullptr, nullptr,
                                                                     n, t, 0.f, 0.f, 0.f, 0.f, 1.f, 1.f);
    CUTB_CUDA_OK(cudaGetLastError());
    return true;
}

CUTB_API bool cutb_conv3d_forward(const void* d_in, const void* d_wf, const float* d_bias, void* d_out, unsigned X,
                                  unsigned Y, unsigned Z, unsigned nb, unsigned cin, unsigned cout, int relu,
                                  int* d_status, void* stream)
{
    ConvFwdArgs a{};
    a.shape = {(int)X, (int)Y, (int)Z, (int)nb};
    a.cin = (int)cin;
    a.cout = (int)cout;
    a.in = (const __nv_bfloat16*)d_in;
    a.wf = (const __nv_bfloat16*)d_wf;
    a.bias = d_bias;
    a.out = (__nv_bfloat16*)d_out;
    a.out_cb_total = (int)cout / 8;
    a.epilogue = relu ? kEpiBiasRelu : kEpiBias;
    a.status = d_status;
    return conv3d_forward(a, (cudaStream_t)stream);
}

CUTB_API bool cutb_conv3d_weight_grad(const void* d_in, const void* d_dout, float* d_dw, unsigned X, unsigned Y,
                                      unsigned Z, unsigned nb, unsigned cin, unsigned cout, int* d_status,
                                      void* stream)
{
    ConvWgradArgs a{};
    a.shape = {(int)X, (int)Y, (int)Z, (int)nb};
    a.cin = (int)cin;
    a.cout = (int)cout;
    a.in = (const __nv_bfloat16*)d_in;
    a.dout = (const __nv_bfloat16*)d_dout;
    a.dw = d_dw;
    a.status = d_status;
    return conv3d_wgrad(a, (cudaStream_t)stream);
}

}  // extern "C"
