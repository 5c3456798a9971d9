/*
 * Extra exports of the CPU build of the upstream sources (TEST INFRASTRUCTURE ONLY; see
 * oracle/Makefile.ref). The upstream entry points themselves (beamform_i16_matlab,
 * init_cuda_configuration, cuda_decode, cuda_hilbert, ...) are exported by the upstream code.
 */
#include "rf_processing/hadamard/hadamard_decoder.h"
#include "image_processing/image_processor.h"

extern "C" __attribute__((visibility("default"))) int ref_encoding_matrix(unsigned n, int ordering, float* out)
{
    // hadamard_decoder.cpp:110-189 writes the matrix to "device" memory, host memory here.
    return decoding::HadamardDecoder::generate_hadamard(out, n, (EncodingMatrix)ordering) ? 0 : -1;
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
