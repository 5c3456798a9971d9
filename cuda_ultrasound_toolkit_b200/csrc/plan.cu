// cutb_plan: everything derived from one CudaBeamformerParameters block, and the
// device-resident stage entry points of include/cuda_toolkit_b200.h.
//
// The plan plays the role of the upstream RfProcessor + Beamformer singletons
// (cuda_toolkit/src/rf_processing/rf_processor.cpp:20-71, beamformer/beamformer.cu:100-137):
// it validates the dimensions, builds the decode transform, uploads the channel map,
// precomputes the match-filter spectrum and the delay-and-sum constants, and owns the
// intermediate buffers. Unlike upstream, nothing is re-planned or re-uploaded per frame,
// no stage synchronises the device, and every stage takes an explicit stream.
#include "plan.h"

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

namespace cutb {

// ---- error state and logging ---------------------------------------------------------------
namespace {
thread_local int g_error = CUTB_OK;
thread_local std::string g_message;
std::atomic<int> g_fail_after{-1};
}  // namespace

int log_level()
{
    static int level = [] {
        const char* e = std::getenv("CUTB_LOG");
        return e ? std::atoi(e) : 1;
    }();
    return level;
}

void set_error(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = code;
    g_message = buf;
    if (log_level() >= 1) std::fprintf(stderr, "[cuda_toolkit_b200] %s\n", buf);
}

void log_info(const char* fmt, ...)
{
    if (log_level() < 2) return;
    va_list ap;
    va_start(ap, fmt);
    std::fprintf(stderr, "[cuda_toolkit_b200] ");
    std::vfprintf(stderr, fmt, ap);
    std::fprintf(stderr, "\n");
    va_end(ap);
}

cudaError_t device_alloc(void** ptr, size_t bytes)
{
    *ptr = nullptr;
    int left = g_fail_after.load();
    if (left == 0) return cudaErrorMemoryAllocation;
    if (left > 0) g_fail_after.compare_exchange_strong(left, left - 1);
    return cudaMalloc(ptr, bytes);
}

void device_free(void* ptr)
{
    if (ptr) cudaFree(ptr);
}

// ---- plan construction ----------------------------------------------------------------------
namespace {

template <class T>
bool upload(T** dst, const T* src, size_t count)
{
    void* p = nullptr;
    cudaError_t e = device_alloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        set_error(CUTB_ERR_ALLOCATION, "Device allocation of %zu bytes failed: %s", count * sizeof(T),
                  cudaGetErrorString(e));
        return false;
    }
    *dst = (T*)p;
    CUTB_CUDA_OK(cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice));
    return true;
}

bool alloc_bytes(void** dst, size_t bytes)
{
    cudaError_t e = device_alloc(dst, bytes);
    if (e != cudaSuccess) {
        set_error(CUTB_ERR_ALLOCATION, "Device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return false;
    }
    return true;
}

}  // namespace

bool FrontEnd::init(const uint32_t raw_dims[2], const uint32_t dec_dims[3], int encoding)
{
    release();
    R0 = raw_dims[0];
    R1 = raw_dims[1];
    S = dec_dims[0];
    C = dec_dims[1];
    T = dec_dims[2];
    // rf_processor.cpp:26-34 (sample and channel counts positive and int32-sized).
    CUTB_REQUIRE(S > 0 && C > 0 && T > 0 && (uint64_t)C * T < (1ull << 31) && S < (1u << 30),
                 CUTB_ERR_INVALID_ARGUMENT, "Invalid dimensions for RF data: %u samples, %u x %u channels.", S, C, T);
    CUTB_REQUIRE(C <= MAX_CHANNEL_COUNT, CUTB_ERR_INVALID_ARGUMENT, "Channel count %u exceeds %d.", C,
                 MAX_CHANNEL_COUNT);
    CUTB_REQUIRE((uint64_t)T * S <= R0, CUTB_ERR_INVALID_ARGUMENT,
                 "Raw rows hold %u samples, fewer than transmits*samples = %llu.", R0, (unsigned long long)T * S);
    CUTB_REQUIRE(R1 > 0 && R1 <= 65536, CUTB_ERR_INVALID_ARGUMENT, "Invalid raw channel count %u.", R1);
    CUTB_REQUIRE(T <= 65535, CUTB_ERR_INVALID_ARGUMENT, "Transmit count %u too large.", T);

    dec.encoding = encoding;
    dec.args = DecodeArgs{};
    dec.args.R0 = R0;
    dec.args.S = S;
    dec.args.C = C;
    dec.args.T = T;
    dec.args.alpha = 1.f;
    std::vector<uint16_t> out_row(T);
    for (uint32_t t = 0; t < T; ++t) out_row[t] = (uint16_t)t;
    if (encoding != NONE) {
        EncodingInfo info;
        if (!build_encoding(T, encoding, info)) return false;
        unsigned R, L;
        CUTB_REQUIRE(plan_decode_split(T, info.base, R, L), CUTB_ERR_UNSUPPORTED, "No decode split for %u transmits.",
                     T);
        dec.base = info.base;
        dec.R = R;
        dec.args.L = L;
        dec.args.G = 32 / L;
        dec.args.alpha = 1.0f / (float)T;  // hadamard_decoder.cpp:65
        out_row = info.natural_to_output;
    }
    if (!upload(&d_out_row, out_row.data(), out_row.size())) return false;
    dec.args.out_row = d_out_row;
    if (!alloc_bytes((void**)&d_map, MAX_CHANNEL_COUNT * sizeof(int16_t))) return false;
    map_set = false;
    return set_filter(nullptr, 0);
}

bool FrontEnd::set_channel_mapping(const int16_t* map, size_t count)
{
    CUTB_REQUIRE(d_map != nullptr, CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(map != nullptr && count >= C, CUTB_ERR_INVALID_ARGUMENT, "Channel mapping needs %u entries.", C);
    for (uint32_t c = 0; c < C; ++c)
        CUTB_REQUIRE(map[c] >= 0 && (uint32_t)map[c] < R1, CUTB_ERR_INVALID_ARGUMENT,
                     "Channel mapping entry %u = %d outside [0, %u).", c, (int)map[c], R1);
    CUTB_CUDA_OK(cudaMemcpy(d_map, map, C * sizeof(int16_t), cudaMemcpyHostToDevice));
    dec.args.map = d_map;
    map_set = true;
    return true;
}

bool FrontEnd::set_filter(const float* taps, uint32_t ntaps)
{
    CUTB_REQUIRE(d_out_row != nullptr, CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(ntaps <= S, CUTB_ERR_INVALID_ARGUMENT, "Match filter longer (%u) than the sample count (%u).",
                 ntaps, S);
    fft_ok = hilbert_supported_length(S);
    if (!fft_ok) return true;  // decode still works; the Hilbert stage reports the length
    std::vector<float> tw, weight;
    if (!build_hilbert_tables(S, taps, ntaps, tw, weight)) return false;
    if (!d_tables && !alloc_bytes((void**)&d_tables, 3 * tw.size() * sizeof(float))) return false;
    CUTB_CUDA_OK(cudaMemcpy(d_tables, tw.data(), tw.size() * sizeof(float), cudaMemcpyHostToDevice));
    CUTB_CUDA_OK(
        cudaMemcpy(d_tables + tw.size(), weight.data(), weight.size() * sizeof(float), cudaMemcpyHostToDevice));
    hil.rows = (uint64_t)T * C;
    hil.n = S;
    hil.log_n = 0;
    while ((1u << hil.log_n) < tw.size() / 2) ++hil.log_n;
    hil.twiddle = d_tables;
    hil.weight = d_tables + tw.size();  // 16-byte aligned: tw.size() is a multiple of 32
    return true;
}

bool FrontEnd::enable_tc_decode(int* status)
{
    CUTB_REQUIRE(d_out_row != nullptr, CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(dec.encoding != NONE, CUTB_ERR_UNSUPPORTED, "Tensor-core decode needs a Hadamard or Walsh code.");
    CUTB_REQUIRE(decode_tc_supported(T, S, R0), CUTB_ERR_UNSUPPORTED,
                 "Tensor-core decode needs 32..256 transmits in steps of 32 and rows of 8-sample multiples "
                 "(T = %u, S = %u, R0 = %u).", T, S, R0);
    std::vector<int8_t> H((size_t)T * T), image;
    if (!cutb_encoding_matrix(T, dec.encoding, (signed char*)H.data())) return false;
    build_decode_tc_image(H.data(), T, image);
    if (!upload(&d_tc_image, image.data(), image.size())) return false;
    d_status = status;
    return true;
}

bool FrontEnd::enable_bandpass(uint32_t S_complex, double fd_over_fs, const float* taps, uint32_t ntaps)
{
    CUTB_REQUIRE(d_out_row != nullptr, CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(S == 2 * S_complex, CUTB_ERR_INVALID_ARGUMENT, "Bandpass rows hold IQ pairs.");
    CUTB_REQUIRE(std::isfinite(fd_over_fs), CUTB_ERR_INVALID_ARGUMENT, "Demodulation frequency must be finite.");
    CUTB_REQUIRE(ntaps <= S_complex, CUTB_ERR_INVALID_ARGUMENT, "Filter longer (%u) than the row (%u).", ntaps,
                 S_complex);
    device_free(d_fir);
    d_fir = nullptr;
    if (ntaps && !upload(&d_fir, taps, ntaps)) return false;
    bandpass = true;
    demod_args.rows = (uint64_t)T * C;
    demod_args.S = (int)S_complex;
    demod_args.L = (int)ntaps;
    demod_args.taps = d_fir;
    demod_args.fd_over_fs = fd_over_fs;
    return true;
}

bool FrontEnd::decode(const void* d_raw, int data_type, float* d_out, unsigned out_stride, cudaStream_t st)
{
    CUTB_REQUIRE(d_out_row != nullptr, CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(map_set, CUTB_ERR_NOT_INITIALIZED, "Channel mapping not set.");
    CUTB_REQUIRE(data_type == TYPE_I16 || data_type == TYPE_F32, CUTB_ERR_UNSUPPORTED,
                 "Data converter: Unsupported input data type %d.", data_type);
    CUTB_REQUIRE(out_stride == 1 || out_stride == 2, CUTB_ERR_INVALID_ARGUMENT, "Output stride must be 1 or 2.");
    CUTB_REQUIRE(d_raw && d_out, CUTB_ERR_INVALID_ARGUMENT, "Null device buffer.");
    if (d_tc_image && data_type == TYPE_I16) {
        DecodeTcArgs a{};
        a.R0 = R0;
        a.S = S;
        a.C = C;
        a.T = T;
        a.map = d_map;
        a.alpha = dec.args.alpha;
        a.out = d_out;
        a.status = d_status;
        return launch_decode_tc(a, d_tc_image, d_raw, out_stride, st);
    }
    return launch_decode(dec, d_raw, data_type, d_out, out_stride, st);
}

bool FrontEnd::hilbert(const float* d_in, unsigned in_stride, void* d_iq, bool bf16, cudaStream_t st)
{
    CUTB_REQUIRE(d_out_row != nullptr, CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    if (bandpass) {
        CUTB_REQUIRE(in_stride == 1, CUTB_ERR_INVALID_ARGUMENT, "Bandpass rows are read packed.");
        CUTB_REQUIRE(d_in && d_iq, CUTB_ERR_INVALID_ARGUMENT, "Null device buffer.");
        return launch_demod_fir(demod_args, d_in, d_iq, bf16, st);
    }
    CUTB_REQUIRE(fft_ok && d_tables != nullptr, CUTB_ERR_UNSUPPORTED,
                 "Sample count %u not supported by the FFT (powers of two up to %u, other lengths up to %u).", S,
                 kMaxHilbertLength, kMaxHilbertLength / 2);
    CUTB_REQUIRE(in_stride == 1 || in_stride == 2, CUTB_ERR_INVALID_ARGUMENT, "Input stride must be 1 or 2.");
    CUTB_REQUIRE(d_in && d_iq, CUTB_ERR_INVALID_ARGUMENT, "Null device buffer.");
    HilbertArgs a = hil;
    a.in_stride = in_stride;
    return launch_hilbert(a, d_in, d_iq, bf16, st);
}

void FrontEnd::release()
{
    device_free(d_tc_image);
    d_tc_image = nullptr;
    device_free(d_fir);
    d_fir = nullptr;
    bandpass = false;
    device_free(d_map);
    device_free(d_out_row);
    device_free(d_tables);
    d_map = nullptr;
    d_out_row = nullptr;
    d_tables = nullptr;
    map_set = false;
    fft_ok = false;
}

}  // namespace cutb

using namespace cutb;

// ---- C ABI ------------------------------------------------------------------------------------
extern "C" {

CUTB_API int cutb_last_error(void) { return g_error; }
CUTB_API const char* cutb_last_error_message(void) { return g_message.c_str(); }
CUTB_API void cutb_clear_error(void)
{
    g_error = CUTB_OK;
    g_message.clear();
}
CUTB_API int cutb_version(void) { return (1 << 16) | 0; }
CUTB_API void cutb_debug_fail_allocations_after(int after) { g_fail_after.store(after); }

CUTB_API cutb_plan* cutb_plan_create(const CudaBeamformerParameters* bp, const cutb_options* options)
{
    if (!bp) {
        set_error(CUTB_ERR_INVALID_ARGUMENT, "cutb_plan_create: null parameters.");
        return nullptr;
    }
    auto* plan = new cutb_plan();
    if (!plan->build(*bp, options)) {
        delete plan;
        return nullptr;
    }
    return plan;
}

CUTB_API void cutb_plan_destroy(cutb_plan* plan) { delete plan; }

CUTB_API size_t cutb_plan_raw_bytes(const cutb_plan* p) { return p ? p->raw_bytes : 0; }
CUTB_API size_t cutb_plan_iq_bytes(const cutb_plan* p) { return p ? p->iq_bytes : 0; }
CUTB_API size_t cutb_plan_volume_bytes(const cutb_plan* p) { return p ? p->vol_bytes : 0; }
CUTB_API int cutb_plan_last_launch_count(const cutb_plan* p) { return p ? p->launches : -1; }

CUTB_API bool cutb_decode(cutb_plan* p, const void* d_raw, size_t raw_bytes, float* d_out, uint out_stride,
                          void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    CUTB_REQUIRE(raw_bytes >= p->raw_bytes, CUTB_ERR_INVALID_ARGUMENT, "Raw buffer holds %zu bytes, need %zu.",
                 raw_bytes, p->raw_bytes);
    p->launches = 0;
    if (!p->fe.decode(d_raw, p->data_type, d_out, out_stride, (cudaStream_t)stream)) return false;
    p->launches = 1;
    return true;
}

CUTB_API bool cutb_hilbert(cutb_plan* p, const float* d_in, uint in_stride, void* d_iq, void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    p->launches = 0;
    if (!p->fe.hilbert(d_in, in_stride, d_iq, p->iq_bf16, (cudaStream_t)stream)) return false;
    p->launches = 1;
    return true;
}

CUTB_API bool cutb_das(cutb_plan* p, const void* d_iq, void* d_volume, void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    CUTB_REQUIRE(d_iq && d_volume, CUTB_ERR_INVALID_ARGUMENT, "Null device buffer.");
    p->launches = 0;
    return launch_das(p->das, d_iq, p->iq_bf16, d_volume, (cudaStream_t)stream, &p->launches);
}

CUTB_API bool cutb_plan_das_tile_shape(const cutb_plan* p, uint shape[3])
{
    CUTB_REQUIRE(p && shape, CUTB_ERR_INVALID_ARGUMENT, "Null argument.");
    int s[3];
    das_tile_shape(p->das, s);
    for (int i = 0; i < 3; ++i) shape[i] = (uint)s[i];
    return true;
}

CUTB_API bool cutb_das_zslab(cutb_plan* p, const void* d_iq, void* d_slab, uint z0, uint z1, void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    CUTB_REQUIRE(d_iq && d_slab, CUTB_ERR_INVALID_ARGUMENT, "Null device buffer.");
    CUTB_REQUIRE(das_staged(p->das), CUTB_ERR_UNSUPPORTED,
                 "Z-slabs need the staged delay-and-sum (not the one-thread-per-voxel kernel).");
    int shape[3];
    das_tile_shape(p->das, shape);
    const uint Z = (uint)p->das.Z, tz = (uint)shape[2];
    CUTB_REQUIRE(z0 < z1 && z1 <= Z && z0 % tz == 0 && (z1 % tz == 0 || z1 == Z), CUTB_ERR_INVALID_ARGUMENT,
                 "Z-slab [%u, %u) must lie in [0, %u) with both ends on the tile depth %u (or the end at %u).", z0, z1,
                 Z, tz, Z);
    DasArgs a = p->das;
    a.z_tile0 = (int)(z0 / tz);
    a.z_tiles = (int)div_up(z1 - z0, tz);
    a.z_out0 = (int)z0;
    p->launches = 0;
    return launch_das(a, d_iq, p->iq_bf16, d_slab, (cudaStream_t)stream, &p->launches);
}

CUTB_API bool cutb_das_tiles(cutb_plan* p, const void* d_iq, void* d_volume, const int* tiles, uint ntiles,
                             uint splits, void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    CUTB_REQUIRE(d_iq && d_volume && tiles && ntiles > 0, CUTB_ERR_INVALID_ARGUMENT, "Null or empty argument.");
    CUTB_REQUIRE(p->das.seq == HERCULES && !p->das.apply_cf, CUTB_ERR_UNSUPPORTED,
                 "Tile-list delay-and-sum supports HERCULES without coherence factor.");
    CUTB_REQUIRE(splits >= 1 && splits <= 4096 && ntiles <= (1u << 24), CUTB_ERR_INVALID_ARGUMENT,
                 "splits must be 1..4096.");
    int shape[3];
    das_tile_shape(p->das, shape);
    const long long total = (long long)div_up(p->das.X, shape[0]) * div_up(p->das.Y, shape[1]) *
                            div_up(p->das.Z, shape[2]);
    for (uint i = 0; i < ntiles; ++i)
        CUTB_REQUIRE(tiles[i] >= 0 && tiles[i] < total, CUTB_ERR_INVALID_ARGUMENT, "Tile id %d outside 0..%lld.",
                     tiles[i], total - 1);
    cudaStream_t st = (cudaStream_t)stream;
    if (ntiles > p->tiles_capacity) {
        device_free(p->d_tiles);
        p->d_tiles = nullptr;
        p->tiles_capacity = 0;
        if (!alloc_bytes((void**)&p->d_tiles, sizeof(int) * ntiles)) return false;
        p->tiles_capacity = ntiles;
    }
    CUTB_CUDA_OK(cudaMemcpyAsync(p->d_tiles, tiles, sizeof(int) * ntiles, cudaMemcpyHostToDevice, st));
    CUTB_CUDA_OK(cudaMemsetAsync(d_volume, 0, p->vol_bytes, st));
    DasArgs a = p->das;
    a.tiles = p->d_tiles;
    a.ntiles = (int)ntiles;
    a.splits = (int)splits;
    p->launches = 0;
    return launch_das(a, d_iq, p->iq_bf16, d_volume, st, &p->launches);
}

CUTB_API bool cutb_plan_check(cutb_plan* p, void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    int status = 0;
    CUTB_CUDA_OK(cudaMemcpyAsync(&status, p->d_status, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CUTB_CUDA_OK(cudaStreamSynchronize((cudaStream_t)stream));
    if (status) {
        CUTB_CUDA_OK(cudaMemsetAsync(p->d_status, 0, sizeof(int), (cudaStream_t)stream));
        set_error(CUTB_ERR_TIMEOUT, "A device-side wait of the delay-and-sum kernel gave up (status %#x).", status);
        return false;
    }
    return true;
}

CUTB_API bool cutb_debug_das_skip_stage(cutb_plan* p, int stage, long long wait_limit_cycles)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    CUTB_REQUIRE(stage >= -1 && wait_limit_cycles >= 0, CUTB_ERR_INVALID_ARGUMENT,
                 "Stage must be -1 (off) or a stage index, the wait limit non-negative.");
    CUTB_REQUIRE(das_staged(p->das), CUTB_ERR_UNSUPPORTED,
                 "Only the staged delay-and-sum has bounded waits (not the one-thread-per-voxel kernel).");
    p->das.debug_skip = stage + 1;
    p->das.wait_limit = wait_limit_cycles;
    return true;
}

CUTB_API bool cutb_beamform(cutb_plan* p, const void* d_raw, size_t raw_bytes, void* d_volume, void* stream)
{
    CUTB_REQUIRE(p, CUTB_ERR_INVALID_ARGUMENT, "Null plan.");
    CUTB_REQUIRE(raw_bytes >= p->raw_bytes, CUTB_ERR_INVALID_ARGUMENT, "Raw buffer holds %zu bytes, need %zu.",
                 raw_bytes, p->raw_bytes);
    CUTB_REQUIRE(d_raw && d_volume, CUTB_ERR_INVALID_ARGUMENT, "Null device buffer.");
    cudaStream_t st = (cudaStream_t)stream;
    p->launches = 0;
    if (!p->ensure_buffers()) return false;
    if (!p->fe.decode(d_raw, p->data_type, p->d_decoded, 1, st)) return false;
    if (!p->fe.hilbert(p->d_decoded, 1, p->d_iq, p->iq_bf16, st)) return false;
    p->launches = 2;
    return launch_das(p->das, p->d_iq, p->iq_bf16, d_volume, st, &p->launches);
}

}  // extern "C"

// ---- plan object ----------------------------------------------------------------------------------
bool cutb_plan::build(const CudaBeamformerParameters& params, const cutb_options* options)
{
    bp = params;
    if (options) opt = *options;
    iq_bf16 = opt.iq_bf16 != 0;
    // cuda_toolkit.cpp:153-182 runs the RF front end for SAMPLE_NORMAL only; bandpass IQ pairs
    // take the demodulation path of RfProcessor::convert_demod here (see bandpass.cu).
    CUTB_REQUIRE(bp.sample_type == SAMPLE_NORMAL || bp.sample_type == SAMPLE_BANDPASS, CUTB_ERR_UNSUPPORTED,
                 "Unsupported sample type: %d", (int)bp.sample_type);
    const bool bandpass = bp.sample_type == SAMPLE_BANDPASS;
    data_type = bp.data_type;
    CUTB_REQUIRE(data_type == TYPE_I16 || data_type == TYPE_F32, CUTB_ERR_UNSUPPORTED,
                 "Data converter: Unsupported input data type %d.", data_type);
    CUTB_REQUIRE(bp.decode == NONE || bp.decode == HADAMARD || bp.decode == WALSH, CUTB_ERR_INVALID_ARGUMENT,
                 "Invalid decode value %d.", (int)bp.decode);
    const uint32_t raw_dims[2] = {bp.rf_raw_dim[0], bp.rf_raw_dim[1]};
    CUTB_REQUIRE(!bandpass || bp.dec_data_dim[0] <= (1u << 29), CUTB_ERR_INVALID_ARGUMENT, "Too many samples.");
    const uint32_t dec_dims[3] = {bandpass ? 2 * bp.dec_data_dim[0] : bp.dec_data_dim[0], bp.dec_data_dim[1],
                                  bp.dec_data_dim[2]};
    if (!fe.init(raw_dims, dec_dims, bp.decode)) return false;
    if (!fe.set_channel_mapping(bp.channel_mapping, MAX_CHANNEL_COUNT)) return false;
    CUTB_REQUIRE(bp.filter_length <= MAX_FILTER_LENGTH, CUTB_ERR_INVALID_ARGUMENT, "Filter length %u exceeds %d.",
                 bp.filter_length, MAX_FILTER_LENGTH);
    if (bandpass) {
        if (!fe.enable_bandpass(bp.dec_data_dim[0], (double)bp.center_frequency / (double)bp.sampling_frequency,
                                bp.rf_filter, bp.filter_length))
            return false;
    } else if (!fe.set_filter(bp.rf_filter, bp.filter_length)) {
        return false;
    }
    if (!derive_das(bp, das)) return false;
    CUTB_REQUIRE(opt.das_tile >= 0 && opt.das_tile <= 3, CUTB_ERR_INVALID_ARGUMENT, "Unknown tile id %d.",
                 opt.das_tile);
    CUTB_REQUIRE(opt.das_tile != 3 || das.seq == RCA_TPW || das.seq == UFORCES, CUTB_ERR_INVALID_ARGUMENT,
                 "The one-thread-per-voxel delay-and-sum (tile 3) serves TPW and UFORCES.");
    das.tile = opt.das_tile;
    CUTB_REQUIRE(opt.das_schedule >= 0 && opt.das_schedule <= 2, CUTB_ERR_INVALID_ARGUMENT,
                 "Unknown delay-and-sum schedule %d.", opt.das_schedule);
    das.schedule = opt.das_schedule;
    CUTB_REQUIRE(opt.das_rows_per_stage >= 0 && opt.das_rows_per_stage <= 8, CUTB_ERR_INVALID_ARGUMENT,
                 "Rows per delay-and-sum stage must be 1..8 (0: 8), not %d.", opt.das_rows_per_stage);
    das.rows_per_stage = opt.das_rows_per_stage;
    if (das.seq == RCA_TPW) {  // beamformer.cu:439-443: angle of transmit t in foci[t][2], radians
        std::vector<float> angles(das.T);
        for (int t = 0; t < das.T; ++t) angles[t] = bp.foci[3 * t + 2];
        if (!upload(&d_angles, angles.data(), angles.size())) return false;
        das.angles = d_angles;
    } else if (das.seq == UFORCES) {
        if (!upload(&d_elems, bp.sparse_elements, (size_t)das.T)) return false;
        das.elems = d_elems;
    }

    const size_t esize = data_type == TYPE_I16 ? 2 : 4;
    raw_bytes = (size_t)bp.rf_raw_dim[0] * bp.rf_raw_dim[1] * esize;
    const size_t samples = (size_t)bp.dec_data_dim[0] * bp.dec_data_dim[1] * bp.dec_data_dim[2];
    iq_bytes = samples * (iq_bf16 ? 4 : 8);
    vol_bytes = (size_t)bp.output_points[0] * bp.output_points[1] * bp.output_points[2] * 8;
    decoded_bytes = samples * sizeof(float) * (bandpass ? 2 : 1);
    if (!alloc_bytes((void**)&d_status, sizeof(int))) return false;
    CUTB_CUDA_OK(cudaMemset(d_status, 0, sizeof(int)));
    das.status = d_status;
    if (opt.decode_tc && !fe.enable_tc_decode(d_status)) return false;
    if (das_staged(das)) {
        // Scratch of the staged delay-and-sum for partial sums of tiles split over several CTAs.
        int dev = 0, sms = 0, counts[3];
        CUTB_CUDA_OK(cudaGetDevice(&dev));
        CUTB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        das_grid_tiles(das, counts);
        const long long tiles = (long long)counts[0] * counts[1] * counts[2];
        // stream-K beyond one wave (on request); the sequences other than HERCULES split a small
        // volume's tiles or a partial last wave
        if ((das.schedule == 2 && tiles > sms) || (das.schedule == 0 && das.seq != HERCULES)) {
            const int pairs = sms * kStreamPairsPerSm;
            if (!alloc_bytes((void**)&d_sk_partials, sizeof(float4) * 2 * kStreamTileVoxels * (size_t)pairs))
                return false;
            if (!alloc_bytes((void**)&d_sk_counters, sizeof(int) * (size_t)pairs)) return false;
            CUTB_CUDA_OK(cudaMemset(d_sk_counters, 0, sizeof(int) * (size_t)pairs));
            das.sk_partials = d_sk_partials;
            das.sk_counters = d_sk_counters;
            das.sk_capacity = pairs;
        }
        if (!prepare_das(das, iq_bf16)) return false;
    }
    return true;
}

// The intermediate buffers of cutb_beamform, allocated on its first call (plans that only run
// stages on caller buffers, such as the frames of a batch, never allocate them).
bool cutb_plan::ensure_buffers()
{
    if (!d_decoded && !alloc_bytes((void**)&d_decoded, decoded_bytes)) return false;
    if (!d_iq && !alloc_bytes(&d_iq, iq_bytes)) return false;
    return true;
}

cutb_plan::~cutb_plan()
{
    device_free(d_decoded);
    device_free(d_iq);
    device_free(d_status);
    device_free(d_tiles);
    device_free(d_angles);
    device_free(d_elems);
    device_free(d_sk_partials);
    device_free(d_sk_counters);
}
