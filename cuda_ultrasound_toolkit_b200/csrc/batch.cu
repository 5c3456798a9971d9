// Batched beamforming of many frames of uneven size: every frame's front end (decode + Hilbert),
// then the delay-and-sum of the frames that fill the GPU on their own as their own grid launches,
// and ONE persistent delay-and-sum launch per kernel variant over the tiles of all smaller frames;
// optionally captured once into a CUDA graph and replayed.
//
// Why: a small frame (64^3 voxels, 32 x 64 rows) fills a fraction of the 148 SMs and a stream of
// such frames pays a launch and a tail per stage. The persistent kernel takes (frame, tile) work
// items from one device counter, heaviest tiles first (longest-processing-time order), so the
// GPU stays full until the last tile of the last frame; the graph removes per-launch host cost.
// A frame with at least one full wave of tiles (SMs x resident CTAs) gains nothing from that and
// runs the single-frame kernel, which reads its arguments from kernel parameters instead of a
// table indexed at run time (the persistent kernel measured about 6 % slower per tile). The
// delay-and-sum launches alternate between two streams forked from the batch's stream (parallel
// branches in the graph), so one launch's tail overlaps the next launch's first wave.
// Frames keep their own parameter blocks (dimensions, geometry, channel map, match filter);
// frames with identical blocks share one plan (tables), each frame has its own buffers.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "common.cuh"
#include "plan.h"
#include "stages.h"

namespace cutb {
namespace {

struct Group {
    bool short_tile = false, iq_bf16 = false;
    DasArgs like{};
    std::vector<int> frames;              // batch frame indices, at most kDasBatchMaxFrames
    std::vector<int2> items;              // (group-local frame, tile id), heaviest first
    int2* d_items = nullptr;
    int* d_counter = nullptr;
    int grid = 0;
    std::unique_ptr<DasBatchParams> params;
};

bool same_group(const Group& g, const DasArgs& a, bool shrt, bool bf16)
{
    return g.short_tile == shrt && g.iq_bf16 == bf16 && g.like.cubic == a.cubic && g.like.apply_cf == a.apply_cf &&
           g.like.use_apo == a.use_apo && (int)g.frames.size() < kDasBatchMaxFrames;
}

}  // namespace
}  // namespace cutb

using namespace cutb;

struct cutb_batch {
    int n = 0;
    std::vector<cutb_plan*> plans;
    std::vector<int> plan_of;
    std::vector<float*> decoded;
    std::vector<void*> iq;
    std::vector<Group> groups;
    std::vector<int> direct;  // frames whose delay-and-sum is a grid launch of its own
    cudaStream_t own = nullptr, side[2] = {nullptr, nullptr};
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fe = nullptr, ev_side[2] = {nullptr, nullptr};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> g_raw;
    std::vector<void*> g_vol;

    ~cutb_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (ev_fe) cudaEventDestroy(ev_fe);
        for (int k = 0; k < 2; ++k) {
            if (ev_side[k]) cudaEventDestroy(ev_side[k]);
            if (side[k]) cudaStreamDestroy(side[k]);
        }
        if (own) cudaStreamDestroy(own);
        for (auto& g : groups) {
            device_free(g.d_items);
            device_free(g.d_counter);
        }
        for (float* p : decoded) device_free(p);
        for (void* p : iq) device_free(p);
        for (cutb_plan* p : plans) cutb_plan_destroy(p);
    }

    bool build(const CudaBeamformerParameters* bp, const cutb_options* opts, uint count)
    {
        n = (int)count;
        int dev = 0, sms = 148;
        CUTB_CUDA_OK(cudaGetDevice(&dev));
        CUTB_CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        for (int i = 0; i < n; ++i) {
            int found = -1;
            for (size_t k = 0; k < plans.size(); ++k)
                if (!std::memcmp(&plans[k]->bp, &bp[i], sizeof(CudaBeamformerParameters)) &&
                    (!opts || !std::memcmp(&plans[k]->opt, &opts[i], sizeof(cutb_options)))) {
                    found = (int)k;
                    break;
                }
            if (found < 0) {
                cutb_plan* p = cutb_plan_create(&bp[i], opts ? &opts[i] : nullptr);
                if (!p) return false;
                plans.push_back(p);
                found = (int)plans.size() - 1;
            }
            plan_of.push_back(found);
            cutb_plan* p = plans[found];
            CUTB_REQUIRE(p->das.seq == HERCULES, CUTB_ERR_UNSUPPORTED,
                         "Frame %d: batched beamforming supports HERCULES frames.", i);
            CUTB_REQUIRE(p->fe.fft_ok || p->fe.bandpass, CUTB_ERR_UNSUPPORTED,
                         "Frame %d: sample count not supported by the FFT.", i);
            const size_t samples = (size_t)bp[i].dec_data_dim[0] * bp[i].dec_data_dim[1] * bp[i].dec_data_dim[2];
            float* d = nullptr;
            void* q = nullptr;
            if (device_alloc((void**)&d, p->decoded_bytes) != cudaSuccess) {
                set_error(CUTB_ERR_ALLOCATION, "Batch frame %d: decoded buffer allocation failed.", i);
                return false;
            }
            decoded.push_back(d);
            if (device_alloc(&q, samples * (p->iq_bf16 ? 4 : 8)) != cudaSuccess) {
                set_error(CUTB_ERR_ALLOCATION, "Batch frame %d: analytic-signal allocation failed.", i);
                return false;
            }
            iq.push_back(q);
            const DasArgs& a = p->das;
            const bool shrt = das_uses_short_tile(a);
            int t[3], per_sm = 0;
            das_grid_tiles(a, t);
            if (!launch_das_batch(nullptr, nullptr, 0, nullptr, a, p->iq_bf16, shrt, 0, &per_sm, 0)) return false;
            if ((long long)t[0] * t[1] * t[2] >= (long long)sms * std::max(per_sm, 1)) {
                direct.push_back(i);
                continue;
            }
            Group* g = nullptr;
            for (auto& gg : groups)
                if (same_group(gg, a, shrt, p->iq_bf16)) g = &gg;
            if (!g) {
                groups.emplace_back();
                g = &groups.back();
                g->short_tile = shrt;
                g->iq_bf16 = p->iq_bf16;
                g->like = a;
            }
            g->frames.push_back(i);
        }
        for (auto& g : groups) {
            struct Item {
                long long cost;
                int frame, tile;
            };
            std::vector<Item> list;
            for (int k = 0; k < (int)g.frames.size(); ++k) {
                const DasArgs& a = plans[plan_of[g.frames[k]]]->das;
                int t[3];
                das_grid_tiles(a, t);
                const long long cost = (long long)a.T * a.C * a.G;
                for (int id = 0; id < t[0] * t[1] * t[2]; ++id) list.push_back({cost, k, id});
            }
            std::stable_sort(list.begin(), list.end(), [](const Item& x, const Item& y) { return x.cost > y.cost; });
            for (const Item& it : list) g.items.push_back(make_int2(it.frame, it.tile));
            if (device_alloc((void**)&g.d_items, g.items.size() * sizeof(int2)) != cudaSuccess ||
                device_alloc((void**)&g.d_counter, sizeof(int)) != cudaSuccess) {
                set_error(CUTB_ERR_ALLOCATION, "Batch work-list allocation failed.");
                return false;
            }
            CUTB_CUDA_OK(
                cudaMemcpy(g.d_items, g.items.data(), g.items.size() * sizeof(int2), cudaMemcpyHostToDevice));
            int per_sm = 0;
            if (!launch_das_batch(nullptr, nullptr, 0, nullptr, g.like, g.iq_bf16, g.short_tile, 0, &per_sm, 0))
                return false;
            g.grid = std::min<long long>((long long)sms * std::max(per_sm, 1), (long long)g.items.size());
            g.params.reset(new DasBatchParams());
        }
        CUTB_CUDA_OK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
        CUTB_CUDA_OK(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
        CUTB_CUDA_OK(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
        CUTB_CUDA_OK(cudaEventCreateWithFlags(&ev_fe, cudaEventDisableTiming));
        for (int k = 0; k < 2; ++k) {
            CUTB_CUDA_OK(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
            CUTB_CUDA_OK(cudaEventCreateWithFlags(&ev_side[k], cudaEventDisableTiming));
        }
        return true;
    }

    // Every kernel of one run, ordered after `st` and before its end, with no host
    // synchronisation (capturable: the side streams fork from and join back into `st`).
    bool enqueue(const void* const* raw, void* const* vol, cudaStream_t st)
    {
        for (int i = 0; i < n; ++i) {
            cutb_plan* p = plans[plan_of[i]];
            if (!p->fe.decode(raw[i], p->data_type, decoded[i], 1, st)) return false;
            if (!p->fe.hilbert(decoded[i], 1, iq[i], p->iq_bf16, st)) return false;
        }
        CUTB_CUDA_OK(cudaEventRecord(ev_fe, st));
        for (int k = 0; k < 2; ++k) CUTB_CUDA_OK(cudaStreamWaitEvent(side[k], ev_fe, 0));
        int next = 0;
        bool ok = true;
        // Persistent launches first: the small frames' tiles then fill the direct launches' tails.
        for (auto& g : groups) {
            if (!ok) break;
            for (int k = 0; k < (int)g.frames.size(); ++k) {
                const int i = g.frames[k];
                g.params->f[k] = DasFrame{plans[plan_of[i]]->das, iq[i], (float2*)vol[i]};
            }
            cudaStream_t s = side[next++ & 1];
            ok = cudaMemsetAsync(g.d_counter, 0, sizeof(int), s) == cudaSuccess;
            if (!ok) set_error(CUTB_ERR_CUDA, "Batch work counter reset failed.");
            ok = ok && launch_das_batch(g.params.get(), g.d_items, (int)g.items.size(), g.d_counter, g.like,
                                        g.iq_bf16, g.short_tile, g.grid, nullptr, s);
        }
        for (size_t d = 0; ok && d < direct.size(); ++d) {
            cutb_plan* p = plans[plan_of[direct[d]]];
            ok = launch_das(p->das, iq[direct[d]], p->iq_bf16, vol[direct[d]], side[next++ & 1], nullptr);
        }
        // Join both side streams back into `st` even after a failure, so a capture stays joined.
        for (int k = 0; k < 2; ++k) {
            CUTB_CUDA_OK(cudaEventRecord(ev_side[k], side[k]));
            CUTB_CUDA_OK(cudaStreamWaitEvent(st, ev_side[k], 0));
        }
        return ok;
    }

    bool run(const void* const* raw, void* const* vol, bool use_graph, cudaStream_t caller)
    {
        for (int i = 0; i < n; ++i)
            CUTB_REQUIRE(raw[i] && vol[i], CUTB_ERR_INVALID_ARGUMENT, "Frame %d: null device buffer.", i);
        // Work on the batch's own stream, ordered after and before the caller's stream.
        CUTB_CUDA_OK(cudaEventRecord(ev_in, caller));
        CUTB_CUDA_OK(cudaStreamWaitEvent(own, ev_in, 0));
        if (!use_graph) {
            if (!enqueue(raw, vol, own)) return false;
        } else {
            bool same = exec && (int)g_raw.size() == n;
            for (int i = 0; same && i < n; ++i) same = g_raw[i] == raw[i] && g_vol[i] == vol[i];
            if (!same) {
                if (exec) cudaGraphExecDestroy(exec);
                if (graph) cudaGraphDestroy(graph);
                exec = nullptr;
                graph = nullptr;
                CUTB_CUDA_OK(cudaStreamBeginCapture(own, cudaStreamCaptureModeThreadLocal));
                const bool ok = enqueue(raw, vol, own);
                cudaGraph_t gr = nullptr;
                const cudaError_t e = cudaStreamEndCapture(own, &gr);
                if (!ok) {
                    if (gr) cudaGraphDestroy(gr);
                    return false;
                }
                CUTB_CUDA_OK(e);
                graph = gr;
                CUTB_CUDA_OK(cudaGraphInstantiate(&exec, graph, 0));
                g_raw.assign(raw, raw + n);
                g_vol.assign(vol, vol + n);
            }
            CUTB_CUDA_OK(cudaGraphLaunch(exec, own));
        }
        CUTB_CUDA_OK(cudaEventRecord(ev_out, own));
        CUTB_CUDA_OK(cudaStreamWaitEvent(caller, ev_out, 0));
        return true;
    }
};

extern "C" {

CUTB_API cutb_batch* cutb_batch_create(const CudaBeamformerParameters* params, const cutb_options* options,
                                       uint count)
{
    if (!params || count == 0 || count > 4096) {
        set_error(CUTB_ERR_INVALID_ARGUMENT, "Batch needs 1..4096 parameter blocks.");
        return nullptr;
    }
    auto* b = new cutb_batch();
    if (!b->build(params, options, count)) {
        delete b;
        return nullptr;
    }
    return b;
}

CUTB_API void cutb_batch_destroy(cutb_batch* b)
{
    if (b) cudaDeviceSynchronize();
    delete b;
}

CUTB_API bool cutb_batch_run(cutb_batch* b, const void* const* d_raw, void* const* d_volume, int use_graph,
                             void* stream)
{
    CUTB_REQUIRE(b && d_raw && d_volume, CUTB_ERR_INVALID_ARGUMENT, "Null argument.");
    return b->run(d_raw, d_volume, use_graph != 0, (cudaStream_t)stream);
}

CUTB_API bool cutb_batch_check(cutb_batch* b, void* stream)
{
    CUTB_REQUIRE(b, CUTB_ERR_INVALID_ARGUMENT, "Null batch.");
    for (cutb_plan* p : b->plans)
        if (!cutb_plan_check(p, stream)) return false;
    return true;
}

// Kernels one run launches: decode and Hilbert per frame, one delay-and-sum per group of small
// frames and one per frame that fills the GPU on its own.
CUTB_API int cutb_batch_launches_per_run(const cutb_batch* b)
{
    return b ? 2 * b->n + (int)(b->groups.size() + b->direct.size()) : 0;
}

CUTB_API int cutb_batch_das_launches(const cutb_batch* b)
{
    return b ? (int)(b->groups.size() + b->direct.size()) : 0;
}

}  // extern "C"
