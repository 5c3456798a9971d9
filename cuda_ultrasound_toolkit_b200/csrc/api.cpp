// Upstream-compatible entry points: cuda_toolkit::beamform, motion_detection and corr_images, the
// MATLAB wrappers and the buffer-registry C ABI (include/cuda_toolkit.hpp, cuda_toolkit_matlab.h,
// cuda_toolkit_ogl.h).
//
// Mirrors the upstream glue (cuda_toolkit/src/api/cuda_toolkit.cpp:109-199,
// cuda_toolkit_matlab.cpp:9-37, cuda_toolkit_ogl.cpp:105-273): process-global cached
// state, device 0, legacy default stream, synchronous return, bool + stderr errors.
// Differences: sizes of caller spans and registered buffers are validated; the plan is
// rebuilt only when the parameter block changes; OpenGL buffer ids are resolved through a
// registry of plain device pointers (cuda_register_device_buffer) because the target
// machine has no graphics stack.
#include <array>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

#include "../../include/cuda_toolkit.hpp"
#include "../../include/cuda_toolkit_matlab.h"
#include "../../include/cuda_toolkit_ogl.h"
#include "../../include/cuda_toolkit_b200_motion.h"
#include "plan.h"

using namespace cutb;

namespace {

// ---- cuda_toolkit::beamform state (upstream cuda_toolkit.cpp:7-40) ------------------------------
struct BeamformState {
    std::unique_ptr<cutb_plan> plan;
    CudaBeamformerParameters bp{};
    void* d_input = nullptr;
    void* d_output = nullptr;
    size_t input_bytes = 0, output_bytes = 0;

    bool ensure(void** ptr, size_t& have, size_t need)
    {
        if (have == need && *ptr) return true;
        device_free(*ptr);
        *ptr = nullptr;
        have = 0;
        cudaError_t e = device_alloc(ptr, need);
        if (e != cudaSuccess) {
            set_error(CUTB_ERR_ALLOCATION, "Failed to update beamformer buffers (%zu bytes): %s", need,
                      cudaGetErrorString(e));
            return false;
        }
        have = need;
        return true;
    }
    void release()
    {
        plan.reset();
        device_free(d_input);
        device_free(d_output);
        d_input = d_output = nullptr;
        input_bytes = output_bytes = 0;
    }
    ~BeamformState() { release(); }
};

BeamformState& beamform_state()
{
    static BeamformState s;
    return s;
}

std::mutex& api_mutex()
{
    static std::mutex m;
    return m;
}

bool beamform_impl(const uint8_t* in, size_t in_size, uint8_t* out, size_t out_size,
                   const CudaBeamformerParameters& bp)
{
    auto& st = beamform_state();
    CUTB_CUDA_OK(cudaSetDevice(0));  // rf_processor.cpp:47
    if (!st.plan || std::memcmp(&st.bp, &bp, sizeof(bp)) != 0) {
        st.plan.reset();
        cutb_plan* p = cutb_plan_create(&bp, nullptr);
        if (!p) return false;
        st.plan.reset(p);
        st.bp = bp;
    }
    cutb_plan* p = st.plan.get();
    CUTB_REQUIRE(in != nullptr && in_size >= p->raw_bytes, CUTB_ERR_INVALID_ARGUMENT,
                 "Input span holds %zu bytes, rf_raw_dim needs %zu.", in_size, p->raw_bytes);
    CUTB_REQUIRE(out != nullptr && out_size >= p->vol_bytes, CUTB_ERR_INVALID_ARGUMENT,
                 "Output span holds %zu bytes, the volume needs %zu.", out_size, p->vol_bytes);
    if (!st.ensure(&st.d_input, st.input_bytes, p->raw_bytes)) return false;
    if (!st.ensure(&st.d_output, st.output_bytes, p->vol_bytes)) return false;
    CUTB_CUDA_OK(cudaMemcpy(st.d_input, in, p->raw_bytes, cudaMemcpyHostToDevice));  // cuda_toolkit.cpp:132
    if (!cutb_beamform(p, st.d_input, p->raw_bytes, st.d_output, nullptr)) return false;
    CUTB_CUDA_OK(cudaMemcpy(out, st.d_output, p->vol_bytes, cudaMemcpyDeviceToHost));  // cuda_toolkit.cpp:188
    return cutb_plan_check(p, nullptr);
}

// ---- buffer-registry session (upstream cuda_toolkit_ogl.cpp:5-30) ---------------------------------
constexpr uint32_t kMaxBufferCount = 16;

struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct Session {
    FrontEnd fe;
    std::map<uint32_t, Buffer> registry;
    uint32_t raw_id = 0;
    std::array<uint32_t, kMaxBufferCount> rf_ids{};
    uint32_t rf_count = 0;
    bool buffers_init = false;
    std::array<int16_t, MAX_CHANNEL_COUNT> map{};
    bool have_map = false;

    void unregister()
    {
        raw_id = 0;
        rf_ids.fill(0);
        rf_count = 0;
        buffers_init = false;
    }
};

Session& session()
{
    static Session s;
    return s;
}

bool lookup(uint32_t id, Buffer& b)
{
    auto& s = session();
    auto it = s.registry.find(id);
    CUTB_REQUIRE(it != s.registry.end(), CUTB_ERR_INVALID_ARGUMENT, "Buffer id %u is not registered.", id);
    b = it->second;
    return true;
}

}  // namespace

// ---- C++ API -----------------------------------------------------------------------------------
bool cuda_toolkit::beamform(std::span<const uint8_t> input_data, std::span<uint8_t> output_data,
                            const CudaBeamformerParameters& bp)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    return beamform_impl(input_data.data(), input_data.size(), output_data.data(), output_data.size(), bp);
}

namespace {

// Device copies of the host spans of the image entry points, kept between calls.
struct ImageBuffers {
    void* ptr[3] = {nullptr, nullptr, nullptr};
    size_t bytes[3] = {0, 0, 0};
    bool ensure(int i, size_t need)
    {
        if (bytes[i] >= need && ptr[i]) return true;
        device_free(ptr[i]);
        ptr[i] = nullptr;
        bytes[i] = 0;
        const cudaError_t e = device_alloc(&ptr[i], need ? need : 16);
        CUTB_REQUIRE(e == cudaSuccess, CUTB_ERR_ALLOCATION, "Image buffer allocation of %zu bytes failed: %s", need,
                     cudaGetErrorString(e));
        bytes[i] = need;
        return true;
    }
    ~ImageBuffers()
    {
        for (void* p : ptr) device_free(p);
    }
};

ImageBuffers& image_buffers()
{
    static ImageBuffers b;
    return b;
}

}  // namespace

// cuda_toolkit.cpp:201-238: frames copied to the device, one block-matching pass, maps copied back.
bool cuda_toolkit::motion_detection(std::span<const uint8_t> images, std::span<uint8_t> motion_maps,
                                    const NccMotionParameters& params)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    const size_t in = sizeof(float) * (size_t)params.image_dims[0] * params.image_dims[1] * params.frame_count;
    const size_t out =
        4 * sizeof(float) * (size_t)params.motion_grid_dims[0] * params.motion_grid_dims[1] * params.frame_count;
    CUTB_REQUIRE(images.data() && images.size() >= in, CUTB_ERR_INVALID_ARGUMENT,
                 "Input image span holds %zu bytes, %u frames of %u x %u floats need %zu.", images.size(),
                 params.frame_count, params.image_dims[0], params.image_dims[1], in);
    CUTB_REQUIRE(motion_maps.data() && motion_maps.size() >= out, CUTB_ERR_INVALID_ARGUMENT,
                 "Motion map span holds %zu bytes, the maps need %zu.", motion_maps.size(), out);
    CUTB_CUDA_OK(cudaSetDevice(0));
    auto& b = image_buffers();
    if (!b.ensure(0, in) || !b.ensure(1, out)) return false;
    CUTB_CUDA_OK(cudaMemcpy(b.ptr[0], images.data(), in, cudaMemcpyHostToDevice));
    if (!cutb_motion_detection((const float*)b.ptr[0], &params, (float*)b.ptr[1], nullptr)) return false;
    CUTB_CUDA_OK(cudaMemcpy(motion_maps.data(), b.ptr[1], out, cudaMemcpyDeviceToHost));
    return true;
}

// cuda_toolkit.cpp:240-329, with upstream's argument checks and messages.
bool cuda_toolkit::corr_images(std::span<const float> template_image, std::span<const float> source_image,
                               std::span<float> corr_map, const uint template_dims[2], const uint source_dims[2])
{
    std::lock_guard<std::mutex> lock(api_mutex());
    CUTB_REQUIRE(template_dims && source_dims, CUTB_ERR_INVALID_ARGUMENT, "Invalid image dimensions for corr_images.");
    const size_t tw = template_dims[0], th = template_dims[1], sw = source_dims[0], sh = source_dims[1];
    CUTB_REQUIRE(tw && th && sw && sh, CUTB_ERR_INVALID_ARGUMENT, "Invalid image dimensions for corr_images.");
    CUTB_REQUIRE(tw <= sw && th <= sh, CUTB_ERR_INVALID_ARGUMENT,
                 "Template dimensions must be <= source dimensions for corr_images.");
    const size_t nt = tw * th, ns = sw * sh, nc = (sw - tw + 1) * (sh - th + 1);
    CUTB_REQUIRE(template_image.size() >= nt && source_image.size() >= ns, CUTB_ERR_INVALID_ARGUMENT,
                 "Input image spans are smaller than the provided dimensions for corr_images.");
    CUTB_REQUIRE(corr_map.size() >= nc, CUTB_ERR_INVALID_ARGUMENT, "Output corr_map span is too small for corr_images.");
    CUTB_CUDA_OK(cudaSetDevice(0));
    auto& b = image_buffers();
    if (!b.ensure(0, ns * sizeof(float)) || !b.ensure(1, nc * sizeof(float)) || !b.ensure(2, nt * sizeof(float)))
        return false;
    CUTB_CUDA_OK(cudaMemcpy(b.ptr[2], template_image.data(), nt * sizeof(float), cudaMemcpyHostToDevice));
    CUTB_CUDA_OK(cudaMemcpy(b.ptr[0], source_image.data(), ns * sizeof(float), cudaMemcpyHostToDevice));
    if (!cutb_corr_images((const float*)b.ptr[2], (const float*)b.ptr[0], template_dims, source_dims,
                          (float*)b.ptr[1], nullptr))
        return false;
    CUTB_CUDA_OK(cudaMemcpy(corr_map.data(), b.ptr[1], nc * sizeof(float), cudaMemcpyDeviceToHost));
    return true;
}

// ---- C ABI ----------------------------------------------------------------------------------------
extern "C" {

void beamform_i16_matlab(const short* data, CudaBeamformerParameters bp, float* output)
{
    // cuda_toolkit_matlab.cpp:9-22
    const size_t in = (size_t)bp.rf_raw_dim[0] * bp.rf_raw_dim[1] * sizeof(short);
    const size_t out = (size_t)bp.output_points[0] * bp.output_points[1] * bp.output_points[2] * 2 * sizeof(float);
    bp.data_type = TYPE_I16;
    std::lock_guard<std::mutex> lock(api_mutex());
    if (!beamform_impl((const uint8_t*)data, in, (uint8_t*)output, out, bp))
        set_error(cutb_last_error(), "Error: Beamforming failed.");
}

void beamform_f32_matlab(const float* data, CudaBeamformerParameters bp, float* output)
{
    // cuda_toolkit_matlab.cpp:24-37
    const size_t in = (size_t)bp.rf_raw_dim[0] * bp.rf_raw_dim[1] * sizeof(float);
    const size_t out = (size_t)bp.output_points[0] * bp.output_points[1] * bp.output_points[2] * 2 * sizeof(float);
    bp.data_type = TYPE_F32;
    std::lock_guard<std::mutex> lock(api_mutex());
    if (!beamform_impl((const uint8_t*)data, in, (uint8_t*)output, out, bp))
        set_error(cutb_last_error(), "Error: Beamforming failed.");
}

void motion_detect_f32_matlab(const float* images, NCCMotionParameters params, float* motion_maps)
{
    // cuda_toolkit_matlab.cpp:39-52
    const size_t in = sizeof(float) * (size_t)params.image_dims[0] * params.image_dims[1] * params.frame_count;
    const size_t out =
        4 * sizeof(float) * (size_t)params.motion_grid_dims[0] * params.motion_grid_dims[1] * params.frame_count;
    if (!cuda_toolkit::motion_detection(std::span<const uint8_t>((const uint8_t*)images, in),
                                        std::span<uint8_t>((uint8_t*)motion_maps, out), params))
        set_error(cutb_last_error(), "Error: Motion detection failed.");
}

void corr_images_f32_matlab(const float* template_image, const float* source_image, CorrImagesParameters params,
                            float* corr_map)
{
    // cuda_toolkit_matlab.cpp:54-76; sizes follow the dims (0 when the template is larger).
    const size_t nt = (size_t)params.template_dims[0] * params.template_dims[1];
    const size_t ns = (size_t)params.source_dims[0] * params.source_dims[1];
    const bool fits = params.template_dims[0] <= params.source_dims[0] && params.template_dims[1] <= params.source_dims[1];
    const size_t nc = fits ? (size_t)(params.source_dims[0] - params.template_dims[0] + 1) *
                                 (params.source_dims[1] - params.template_dims[1] + 1)
                           : 0;
    if (!cuda_toolkit::corr_images(std::span<const float>(template_image, nt), std::span<const float>(source_image, ns),
                                   std::span<float>(corr_map, nc), params.template_dims, params.source_dims))
        set_error(cutb_last_error(), "Error: Correlation failed.");
}

bool init_cuda_configuration(const uint* input_dims, const uint* decoded_dims)
{
    // cuda_toolkit_ogl.cpp:105-117; the encoding is fixed to HADAMARD (rf_processor.h:29).
    CUTB_REQUIRE(input_dims && decoded_dims, CUTB_ERR_INVALID_ARGUMENT, "Null dimension array.");
    std::lock_guard<std::mutex> lock(api_mutex());
    CUTB_CUDA_OK(cudaSetDevice(0));
    auto& s = session();
    const uint32_t raw[2] = {input_dims[0], input_dims[1]};
    const uint32_t dec[3] = {decoded_dims[0], decoded_dims[1], decoded_dims[2]};
    if (!s.fe.init(raw, dec, HADAMARD)) {
        set_error(cutb_last_error(), "Failed to initialize CUDA session.");
        return false;
    }
    if (s.have_map && !s.fe.set_channel_mapping(s.map.data(), s.map.size())) return false;
    return true;
}

void deinit_cuda_configuration(void)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    auto& s = session();
    s.fe.release();
    s.unregister();
    s.registry.clear();
    s.have_map = false;
    beamform_state().release();
}

bool cuda_register_device_buffer(uint id, void* dptr, size_t bytes)
{
    CUTB_REQUIRE(id != 0, CUTB_ERR_INVALID_ARGUMENT, "Buffer id 0 is reserved.");
    std::lock_guard<std::mutex> lock(api_mutex());
    auto& s = session();
    if (!dptr) {
        s.registry.erase(id);
        return true;
    }
    s.registry[id] = Buffer{dptr, bytes};
    return true;
}

bool register_cuda_buffers(const uint* rf_data_ssbos, uint rf_buffer_count, uint raw_data_ssbo)
{
    // cuda_toolkit_ogl.cpp:127-160
    std::lock_guard<std::mutex> lock(api_mutex());
    auto& s = session();
    s.unregister();
    CUTB_REQUIRE(rf_buffer_count <= kMaxBufferCount, CUTB_ERR_INVALID_ARGUMENT,
                 "Too many RF data buffers. Maximum is %u.", kMaxBufferCount);
    CUTB_REQUIRE(rf_buffer_count == 0 || rf_data_ssbos, CUTB_ERR_INVALID_ARGUMENT, "Null buffer id list.");
    Buffer b;
    if (!lookup(raw_data_ssbo, b)) return false;
    for (uint i = 0; i < rf_buffer_count; ++i) {
        CUTB_REQUIRE(rf_data_ssbos[i] != 0, CUTB_ERR_INVALID_ARGUMENT, "Invalid SSBO at index %u.", i);
        if (!lookup(rf_data_ssbos[i], b)) return false;
    }
    s.raw_id = raw_data_ssbo;
    for (uint i = 0; i < rf_buffer_count; ++i) s.rf_ids[i] = rf_data_ssbos[i];
    s.rf_count = rf_buffer_count;
    s.buffers_init = true;
    return true;
}

bool cuda_set_channel_mapping(const i16 channel_mapping[MAX_CHANNEL_COUNT])
{
    // cuda_toolkit_ogl.cpp:162-175: all 256 entries are copied; the first C are used.
    CUTB_REQUIRE(channel_mapping, CUTB_ERR_INVALID_ARGUMENT, "Null channel mapping.");
    std::lock_guard<std::mutex> lock(api_mutex());
    auto& s = session();
    std::memcpy(s.map.data(), channel_mapping, sizeof(int16_t) * MAX_CHANNEL_COUNT);
    s.have_map = true;
    if (s.fe.ready() && !s.fe.set_channel_mapping(s.map.data(), s.map.size())) {
        set_error(cutb_last_error(), "Failed to set channel mapping.");
        return false;
    }
    return true;
}

bool cuda_set_match_filter(const float* match_filter, uint length)
{
    // cuda_toolkit_ogl.cpp:177-190, rf_processor.cpp:100-116
    std::lock_guard<std::mutex> lock(api_mutex());
    auto& s = session();
    CUTB_REQUIRE(s.fe.ready(), CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(length == 0 || match_filter, CUTB_ERR_INVALID_ARGUMENT, "Null match filter.");
    if (!s.fe.set_filter(match_filter, length)) {
        set_error(cutb_last_error(), "Failed to set match filter.");
        return false;
    }
    return true;
}

bool cuda_decode(size_t input_offset, uint output_buffer_idx)
{
    // cuda_toolkit_ogl.cpp:192-235: int16 input, complex output with the decoded value in .x.
    std::lock_guard<std::mutex> lock(api_mutex());
    auto& s = session();
    CUTB_REQUIRE(s.buffers_init, CUTB_ERR_NOT_INITIALIZED, "OGL buffers not registered.");
    CUTB_REQUIRE(s.fe.ready(), CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(output_buffer_idx < s.rf_count, CUTB_ERR_INVALID_ARGUMENT, "Output buffer index %u >= %u.",
                 output_buffer_idx, s.rf_count);
    Buffer raw, out;
    if (!lookup(s.raw_id, raw) || !lookup(s.rf_ids[output_buffer_idx], out)) return false;
    const size_t offset = input_offset / sizeof(int16_t) * sizeof(int16_t);
    const size_t need_in = (size_t)s.fe.R0 * s.fe.R1 * sizeof(int16_t);
    const size_t need_out = (size_t)s.fe.S * s.fe.C * s.fe.T * 8;
    CUTB_REQUIRE(offset <= raw.bytes && raw.bytes - offset >= need_in, CUTB_ERR_INVALID_ARGUMENT,
                 "Raw buffer too small: %zu bytes after offset %zu, need %zu.", raw.bytes - std::min(offset, raw.bytes),
                 offset, need_in);
    CUTB_REQUIRE(out.bytes >= need_out, CUTB_ERR_INVALID_ARGUMENT, "RF buffer holds %zu bytes, need %zu.", out.bytes,
                 need_out);
    if (!s.fe.decode((const uint8_t*)raw.ptr + offset, TYPE_I16, (float*)out.ptr, 2, nullptr)) {
        set_error(cutb_last_error(), "Failed to decode data.");
        return false;
    }
    CUTB_CUDA_OK(cudaStreamSynchronize(nullptr));
    return true;
}

bool cuda_hilbert(uint input_buffer_idx, uint output_buffer_idx)
{
    // cuda_toolkit_ogl.cpp:237-273: reads .x of the complex input buffer.
    std::lock_guard<std::mutex> lock(api_mutex());
    auto& s = session();
    CUTB_REQUIRE(s.buffers_init, CUTB_ERR_NOT_INITIALIZED, "OGL buffers not registered.");
    CUTB_REQUIRE(s.fe.ready(), CUTB_ERR_NOT_INITIALIZED, "Session not initialized.");
    CUTB_REQUIRE(input_buffer_idx < s.rf_count && output_buffer_idx < s.rf_count, CUTB_ERR_INVALID_ARGUMENT,
                 "Buffer index out of range (%u registered).", s.rf_count);
    Buffer in, out;
    if (!lookup(s.rf_ids[input_buffer_idx], in) || !lookup(s.rf_ids[output_buffer_idx], out)) return false;
    const size_t need = (size_t)s.fe.S * s.fe.C * s.fe.T * 8;
    CUTB_REQUIRE(in.bytes >= need && out.bytes >= need, CUTB_ERR_INVALID_ARGUMENT, "RF buffers need %zu bytes.",
                 need);
    if (!s.fe.hilbert((const float*)in.ptr, 2, out.ptr, false, nullptr)) return false;
    CUTB_CUDA_OK(cudaStreamSynchronize(nullptr));
    return true;
}

}  // extern "C"
