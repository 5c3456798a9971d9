// Server of the out-of-process transfer path: the command socket, the shared-memory segments and
// the message loop with upstream's request handlers (test_app/src/transfer_server.cpp,
// test_app.cpp:42-304), on POSIX primitives.
//
// Kept from upstream: the message layout and order (validate, ACK, run, output at the start of
// the data segment, SUCCESS with the output size, or ERR), one client at a time, a disconnected
// client replaced by the next one, the idle timeout.
// Changed: a failed request answers ERR and the server keeps serving (upstream throws out of its
// loop after answering ERR); a request larger than the data segment answers ERR and keeps
// serving (upstream ends its loop); motion detection answers ERR when it fails (upstream answers
// SUCCESS whatever the result); SVD_FILTER and unknown opcodes answer ERR (upstream logs them and
// never answers, so its client waits until its 20-minute timeout); clients of another user are
// refused (abstract sockets have no file permissions); results are formed in a staging buffer and
// copied to the data segment only while the requesting client is still connected, so a client
// that gave up (timeout) and already placed its next input in the segment does not have that
// input overwritten by the late result.
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <span>
#include <string>

#include <fcntl.h>
#include <poll.h>
#include <sys/mman.h>
#include <sys/socket.h>
#include <sys/stat.h>
#include <sys/un.h>
#include <unistd.h>

#include "../../include/cuda_toolkit.hpp"
#include "../../include/cuda_toolkit_b200_server.h"
#include "common.cuh"

using namespace cutb;

struct cutb_server {
    std::string base, data_name, params_name, sock_name;
    int listen_fd = -1, client_fd = -1;
    uint8_t* data = nullptr;
    size_t data_bytes = 0;
    SharedMemoryParams* params = nullptr;
    cutb_server_handler handler = nullptr;
    void* user = nullptr;
    std::atomic<bool> stop{false};
    bool pinned = false;
    uint8_t* staging = nullptr;  // result buffer, page-locked when a GPU is present
    size_t staging_bytes = 0;
    bool staging_pinned = false;

    ~cutb_server()
    {
        release_staging();
        if (client_fd >= 0) close(client_fd);
        if (listen_fd >= 0) close(listen_fd);
        if (pinned) cudaHostUnregister(data);
        if (data) munmap(data, data_bytes);
        if (params) munmap(params, sizeof(SharedMemoryParams));
        if (!data_name.empty()) shm_unlink(data_name.c_str());
        if (!params_name.empty()) shm_unlink(params_name.c_str());
    }

    static void* create_segment(const std::string& name, size_t bytes)
    {
        shm_unlink(name.c_str());  // a segment left by a previous server
        const int fd = shm_open(name.c_str(), O_CREAT | O_EXCL | O_RDWR, 0600);
        if (fd < 0) return nullptr;
        void* p = MAP_FAILED;
        if (ftruncate(fd, (off_t)bytes) == 0) p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
        close(fd);
        return p == MAP_FAILED ? nullptr : p;
    }

    bool create(const char* name, uint64_t bytes)
    {
        const char* env = getenv("CUDA_TRANSFER_NAME");
        base = name && *name ? name : (env && *env ? env : CUDA_TRANSFER_DEFAULT_NAME);
        CUTB_REQUIRE(base.size() < 80 && base.find('/') == std::string::npos, CUTB_ERR_INVALID_ARGUMENT,
                     "Transfer name '%s' must be shorter than 80 characters, without '/'.", base.c_str());
        data_bytes = bytes ? (size_t)bytes : (size_t)DATA_SMEM_SIZE;
        sock_name = base + COMMAND_SOCKET_SUFFIX;
        listen_fd = socket(AF_UNIX, SOCK_SEQPACKET | SOCK_CLOEXEC, 0);
        CUTB_REQUIRE(listen_fd >= 0, CUTB_ERR_INVALID_ARGUMENT, "Failed to create the command socket: %s",
                     strerror(errno));
        sockaddr_un addr{};
        addr.sun_family = AF_UNIX;
        memcpy(addr.sun_path + 1, sock_name.data(), sock_name.size());
        const socklen_t len = (socklen_t)(offsetof(sockaddr_un, sun_path) + 1 + sock_name.size());
        // The socket name is the lock: a second server of the same name fails here, before it
        // could replace the running server's segments.
        if (bind(listen_fd, (sockaddr*)&addr, len) != 0 || listen(listen_fd, 4) != 0) {
            const int e = errno;
            set_error(CUTB_ERR_INVALID_ARGUMENT, "Failed to set up command socket '%s': %s", sock_name.c_str(),
                      strerror(e));
            return false;
        }
        // Named only now: the destructor removes the segments of these names.
        data_name = "/" + base + DATA_SMEM_SUFFIX;
        params_name = "/" + base + PARAMETERS_SMEM_SUFFIX;
        data = (uint8_t*)create_segment(data_name, data_bytes);
        CUTB_REQUIRE(data, CUTB_ERR_ALLOCATION, "Failed to set up data shared memory '%s' (%zu bytes): %s",
                     data_name.c_str(), data_bytes, strerror(errno));
        params = (SharedMemoryParams*)create_segment(params_name, sizeof(SharedMemoryParams));
        CUTB_REQUIRE(params, CUTB_ERR_ALLOCATION, "Failed to set up parameter shared memory '%s': %s",
                     params_name.c_str(), strerror(errno));
        return true;
    }

    bool respond(CudaCommand op, uint64_t size)
    {
        CommandPipeMessage m;
        memset(&m, 0, sizeof(m));
        m.opcode = op;
        m.data_size = size;
        if (client_fd < 0 || send(client_fd, &m, sizeof(m), MSG_NOSIGNAL) != (ssize_t)sizeof(m)) {
            log_info("Error writing to the command socket: %s", strerror(errno));
            return false;
        }
        return true;
    }

    void drop_client()
    {
        if (client_fd >= 0) close(client_fd);
        client_fd = -1;
    }

    // 1: a command in `m`; 0: idle timeout or stop; -1: socket error.
    int wait_for_command(CommandPipeMessage& m, int idle_timeout_ms)
    {
        const auto start = std::chrono::steady_clock::now();
        while (!stop.load()) {
            if (idle_timeout_ms > 0 &&
                std::chrono::steady_clock::now() - start > std::chrono::milliseconds(idle_timeout_ms)) {
                log_info("Command wait timed out");
                return 0;
            }
            pollfd pfd{client_fd >= 0 ? client_fd : listen_fd, POLLIN, 0};
            const int r = poll(&pfd, 1, 100);
            if (r < 0 && errno != EINTR) return -1;
            if (r <= 0) continue;
            if (client_fd < 0) {
                const int fd = accept4(listen_fd, nullptr, nullptr, SOCK_CLOEXEC);
                if (fd < 0) continue;
                ucred cred{};
                socklen_t cl = sizeof(cred);
                if (getsockopt(fd, SOL_SOCKET, SO_PEERCRED, &cred, &cl) != 0 || cred.uid != getuid()) {
                    log_info("Refused a client of another user");
                    close(fd);
                    continue;
                }
                client_fd = fd;
                continue;
            }
            const ssize_t n = recv(client_fd, &m, sizeof(m), 0);
            if (n == 0 || (n < 0 && errno != EINTR && errno != EAGAIN)) {
                log_info("Client disconnected");
                drop_client();
                continue;
            }
            if (n != (ssize_t)sizeof(m)) {
                log_info("Ignored a %zd-byte message on the command socket", n);
                continue;
            }
            return 1;
        }
        return 0;
    }

    void release_staging()
    {
        if (staging_pinned)
            cudaFreeHost(staging);
        else
            free(staging);
        staging = nullptr;
        staging_bytes = 0;
        staging_pinned = false;
    }

    uint8_t* ensure_staging(size_t bytes, bool want_pinned)
    {
        if (staging && staging_bytes >= bytes && (staging_pinned || !want_pinned)) return staging;
        release_staging();
        const size_t n = bytes ? bytes : 16;
        if (want_pinned && cudaMallocHost((void**)&staging, n) == cudaSuccess) {
            staging_pinned = true;
        } else {
            cudaGetLastError();
            staging = (uint8_t*)malloc(n);
        }
        staging_bytes = staging ? n : 0;
        return staging;
    }

    // The requesting client has not closed its end.
    bool client_alive()
    {
        if (client_fd < 0) return false;
        pollfd pfd{client_fd, POLLRDHUP, 0};
        return poll(&pfd, 1, 0) == 0 || !(pfd.revents & (POLLRDHUP | POLLHUP | POLLERR | POLLNVAL));
    }

    // Result in the staging buffer -> start of the data segment + SUCCESS, if anyone still waits.
    bool deliver(size_t bytes)
    {
        if (!client_alive()) {
            log_info("The client left before its result was ready; result dropped.");
            return true;
        }
        memcpy(data, staging, bytes);
        return respond(SUCCESS, bytes);
    }

    void pin()
    {
        if (!pinned) pinned = cudaHostRegister(data, data_bytes, cudaHostRegisterDefault) == cudaSuccess;
        if (!pinned) cudaGetLastError();
    }

    // TestApp::_handle_beamform_command (test_app.cpp:101-154)
    bool beamform(const CommandPipeMessage& c)
    {
        const CudaBeamformerParameters& bp = params->beamformerParameters;
        respond(ACK, 0);
        const size_t out = (size_t)bp.output_points[0] * bp.output_points[1] * bp.output_points[2] * 2 * sizeof(float);
        if (out > data_bytes) {
            log_info("Error: Output size exceeds shared memory size.");
            return false;
        }
        pin();
        uint8_t* res = ensure_staging(out, true);
        if (!res) return false;
        if (!cuda_toolkit::beamform(std::span<const uint8_t>(data, c.data_size), std::span<uint8_t>(res, out), bp)) {
            log_info("Error: Beamforming failed.");
            return false;
        }
        return deliver(out);
    }

    // TestApp::_handle_motion_detection_command (test_app.cpp:156-212)
    bool motion(const CommandPipeMessage& c)
    {
        const NccMotionParameters& p = params->nccMotionParameters;
        respond(ACK, 0);
        const size_t out = (size_t)p.motion_grid_dims[0] * p.motion_grid_dims[1] * 4 * sizeof(float) * p.frame_count;
        if (out > data_bytes) {
            log_info("Error: Output size exceeds shared memory size.");
            return false;
        }
        pin();
        uint8_t* res = ensure_staging(out, true);
        if (!res) return false;
        if (!cuda_toolkit::motion_detection(std::span<const uint8_t>(data, c.data_size), std::span<uint8_t>(res, out),
                                            p)) {
            log_info("Error: Motion detection failed.");
            return false;
        }
        return deliver(out);
    }

    // TestApp::_handle_corr_images_command (test_app.cpp:214-304)
    bool corr(const CommandPipeMessage& c)
    {
        const CorrImagesParameters p = params->corrImagesParameters;
        if (!p.template_dims[0] || !p.template_dims[1] || !p.source_dims[0] || !p.source_dims[1]) {
            log_info("Error: Invalid corr_images dimensions.");
            return false;
        }
        if (p.template_dims[0] > p.source_dims[0] || p.template_dims[1] > p.source_dims[1]) {
            log_info("Error: Template dimensions must be <= source dimensions.");
            return false;
        }
        const size_t nt = (size_t)p.template_dims[0] * p.template_dims[1];
        const size_t ns = (size_t)p.source_dims[0] * p.source_dims[1];
        const size_t nc = ((size_t)p.source_dims[0] - p.template_dims[0] + 1) *
                          ((size_t)p.source_dims[1] - p.template_dims[1] + 1);
        if (c.data_size != (nt + ns) * sizeof(float)) {
            log_info("Error: Input data size does not match corr_images dimensions.");
            return false;
        }
        if (nc * sizeof(float) > data_bytes) {
            log_info("Error: Output size exceeds shared memory size.");
            return false;
        }
        respond(ACK, 0);
        pin();
        uint8_t* res = ensure_staging(nc * sizeof(float), true);
        if (!res) return false;
        const float* f = reinterpret_cast<const float*>(data);
        if (!cuda_toolkit::corr_images(std::span<const float>(f, nt), std::span<const float>(f + nt, ns),
                                       std::span<float>(reinterpret_cast<float*>(res), nc), p.template_dims,
                                       p.source_dims)) {
            log_info("Error: corr_images failed.");
            return false;
        }
        return deliver(nc * sizeof(float));
    }

    bool custom(const CommandPipeMessage& c)
    {
        respond(ACK, 0);
        uint8_t* res = ensure_staging(data_bytes, false);
        if (!res) return false;
        uint64_t out = 0;
        const int rc = handler((int)c.opcode, params, data, c.data_size, res, data_bytes, &out, user);
        if (rc != 0 || out > data_bytes) return false;
        return deliver(out);
    }

    int serve(int max_commands, int idle_timeout_ms)
    {
        int handled = 0;
        while (max_commands <= 0 || handled < max_commands) {
            CommandPipeMessage c;
            const int w = wait_for_command(c, idle_timeout_ms);
            if (w < 0) {
                set_error(CUTB_ERR_INVALID_ARGUMENT, "Command socket error: %s", strerror(errno));
                stop.store(false);
                return -1;
            }
            if (w == 0) break;
            ++handled;
            if (c.opcode == ACK || c.opcode == ERR || c.opcode == SUCCESS) {
                log_info("Ignored response opcode %d from the client.", (int)c.opcode);
                continue;
            }
            if (c.data_size > data_bytes) {
                log_info("Data size too large: %llu, Max: %zu", c.data_size, data_bytes);
                respond(ERR, 0);
                continue;
            }
            bool ok = false;
            if (c.opcode == BEAMFORM_VOLUME || c.opcode == NCC_MOTION_DETECT || c.opcode == CORR_IMAGES) {
                if (handler)
                    ok = custom(c);
                else if (c.opcode == BEAMFORM_VOLUME)
                    ok = beamform(c);
                else if (c.opcode == NCC_MOTION_DETECT)
                    ok = motion(c);
                else
                    ok = corr(c);
            } else {
                log_info("Unsupported command opcode (%d).", (int)c.opcode);
            }
            if (!ok) respond(ERR, 0);
        }
        stop.store(false);  // a stop request ends one serve call
        return handled;
    }
};

extern "C" {

CUTB_API cutb_server* cutb_server_create(const char* name, uint64_t data_bytes)
{
    auto* s = new cutb_server();
    if (!s->create(name, data_bytes)) {
        delete s;
        return nullptr;
    }
    return s;
}

CUTB_API void cutb_server_set_handler(cutb_server* s, cutb_server_handler handler, void* user)
{
    if (!s) return;
    s->handler = handler;
    s->user = user;
}

CUTB_API int cutb_server_serve(cutb_server* s, int max_commands, int idle_timeout_ms)
{
    if (!s) {
        set_error(CUTB_ERR_INVALID_ARGUMENT, "Null server.");
        return -1;
    }
    return s->serve(max_commands, idle_timeout_ms);
}

CUTB_API void cutb_server_stop(cutb_server* s)
{
    if (s) s->stop.store(true);
}

CUTB_API void cutb_server_destroy(cutb_server* s) { delete s; }

}  // extern "C"
