// Plan and RF front-end state shared by plan.cu and the upstream-compatible ABI (api.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "encoding.h"
#include "stages.h"

namespace cutb {

// Decode + Hilbert state for one set of dimensions: the RfProcessor of upstream
// (cuda_toolkit/src/rf_processing/rf_processor.h:14-73) without the per-call re-planning.
struct FrontEnd {
    uint32_t R0 = 0, R1 = 0, S = 0, C = 0, T = 0;
    DecodeSetup dec;
    HilbertArgs hil{};
    int16_t* d_map = nullptr;
    uint16_t* d_out_row = nullptr;
    float* d_tables = nullptr;  // twiddle | ge | go, 2*S floats each
    bool map_set = false;
    bool fft_ok = false;      // S is a length the FFT kernel supports
    int8_t* d_tc_image = nullptr;  // canonical encoding matrix of the tensor-core decode (null: FWHT)
    bool bandpass = false;         // SAMPLE_BANDPASS: decode 2 S raw samples per row, then demod + FIR
    DemodArgs demod_args{};
    float* d_fir = nullptr;
    int* d_status = nullptr;       // status word the tensor-core decode reports bounded waits in

    bool init(const uint32_t raw_dims[2], const uint32_t dec_dims[3], int encoding);
    bool set_channel_mapping(const int16_t* map, size_t count);
    bool set_filter(const float* taps, uint32_t ntaps);
    bool enable_tc_decode(int* status);
    // Bandpass plans: IQ pairs of `S` complex samples, demodulated at fd / fs and filtered.
    bool enable_bandpass(uint32_t S_complex, double fd_over_fs, const float* taps, uint32_t ntaps);
    bool decode(const void* d_raw, int data_type, float* d_out, unsigned out_stride, cudaStream_t st);
    bool hilbert(const float* d_in, unsigned in_stride, void* d_iq, bool bf16, cudaStream_t st);
    bool ready() const { return d_out_row != nullptr; }
    void release();
    ~FrontEnd() { release(); }
};

}  // namespace cutb

struct cutb_plan {
    CudaBeamformerParameters bp{};
    cutb_options opt{};
    bool iq_bf16 = false;
    int data_type = TYPE_I16;
    cutb::FrontEnd fe;
    cutb::DasArgs das{};
    size_t raw_bytes = 0, iq_bytes = 0, vol_bytes = 0, decoded_bytes = 0;
    float* d_decoded = nullptr;
    void* d_iq = nullptr;
    int* d_status = nullptr;   // device-side error word of the stage kernels
    int* d_tiles = nullptr;    // tile list of cutb_das_tiles
    float* d_angles = nullptr; // RCA_TPW plane-wave angles
    short* d_elems = nullptr;  // UFORCES transmit elements
    float4* d_sk_partials = nullptr;  // stream-K partial sums of the delay-and-sum (large volumes)
    int* d_sk_counters = nullptr;
    uint32_t tiles_capacity = 0;
    int launches = 0;

    bool build(const CudaBeamformerParameters& params, const cutb_options* options);
    bool ensure_buffers();
    ~cutb_plan();
};
