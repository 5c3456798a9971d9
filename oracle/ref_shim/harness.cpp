/*
 * Extra exports of the CPU build of the upstream sources (TEST INFRASTRUCTURE ONLY; see
 * oracle/Makefile.ref). The upstream entry points themselves (beamform_i16_matlab,
 * init_cuda_configuration, cuda_decode, cuda_hilbert, ...) are exported by the upstream code.
 */
#include <span>

#include "rf_processing/hadamard/hadamard_decoder.h"
#include "rf_processing/rf_processor.h"
#include "image_processing/image_processor.h"

extern "C" __attribute__((visibility("default"))) int ref_encoding_matrix(unsigned n, int ordering, float* out)
{
    // hadamard_decoder.cpp:110-189 writes the matrix to "device" memory, host memory here.
    return decoding::HadamardDecoder::generate_hadamard(out, n, (EncodingMatrix)ordering) ? 0 : -1;
}

// RfProcessor::convert_demod (rf_processor.cpp:225-246, data_converter.cu:63-131): bandpass IQ
// pairs -> demodulated, time-domain filtered complex [T][C][S]. No upstream entry point calls it.
extern "C" __attribute__((visibility("default"))) int ref_convert_demod(const void* raw, int data_type, unsigned R0,
                                                                       unsigned R1, unsigned S, unsigned C, unsigned T,
                                                                       const short* map256, float demod_freq,
                                                                       float sample_freq, const float* taps, int ntaps,
                                                                       void* out)
{
    RfProcessor p;
    if (!p.init({R0, R1}, {S, C, T})) return -1;
    if (!p.set_channel_mapping(std::span<const int16_t>(map256, 256))) return -1;
    return p.convert_demod(const_cast<void*>(raw), (cuComplex*)out, (InputDataTypes)data_type, demod_freq,
                           sample_freq, taps, ntaps)
               ? 0
               : -1;
}

// The motion-detection members that cuda_toolkit.cpp references are outside the RF -> volume
// path; these definitions only satisfy the linker and report failure if called.
NppStreamContext ImageProcessor::_create_stream_context(cudaStream_t) { return NppStreamContext{}; }
bool ImageProcessor::corr_images(const PitchedArray<float>&, const PitchedArray<float>&, float*, uint2, uint2)
{
    return false;
}
bool ImageProcessor::ncc_block_match(std::vector<PitchedArray<float>>&, float4*, const NccMotionParameters&)
{
    return false;
}
