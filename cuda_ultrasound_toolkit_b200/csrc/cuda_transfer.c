/*
 * Client of the out-of-process transfer path (libcuda_transfer.so; plain C, no CUDA).
 *
 * Same functions and flow as upstream's client library (test_app/client_lib/cuda_transfer.c:
 * 370-467): map the server's shared memory, write the parameter block and the input, send one
 * CommandPipeMessage, wait for ACK, wait for the result, copy the output. On any failure the
 * shared memory and the socket are released (upstream _cleanup_shared_resources), so the next
 * call reconnects. Differences: the result size announced by the server is checked against the
 * caller's output size before copying, and the status of the last call is kept.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <fcntl.h>
#include <poll.h>
#include <stdarg.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/socket.h>
#include <sys/stat.h>
#include <sys/un.h>
#include <time.h>
#include <unistd.h>

#include "../../include/cuda_transfer.h"

#define RESPONSE_POLL_TIMEOUT_MS 1200000u /* 20 minutes, as upstream */

static SharedMemoryParams* g_params = NULL;
static size_t g_params_bytes = 0;
static void* g_data = NULL;
static size_t g_data_bytes = 0;
static int g_sock = -1;
static int g_status = CUDA_TRANSFER_OK;
static unsigned g_timeout_ms = RESPONSE_POLL_TIMEOUT_MS;

static void report(int code, const char* fmt, ...)
{
    va_list ap;
    g_status = code;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fputc('\n', stderr);
}

static const char* base_name(void)
{
    const char* n = getenv("CUDA_TRANSFER_NAME");
    return (n && *n) ? n : CUDA_TRANSFER_DEFAULT_NAME;
}

static void cleanup_shared_resources(void)
{
    if (g_data) munmap(g_data, g_data_bytes);
    if (g_params) munmap(g_params, g_params_bytes);
    if (g_sock >= 0) close(g_sock);
    g_data = NULL;
    g_params = NULL;
    g_data_bytes = g_params_bytes = 0;
    g_sock = -1;
}

static bool open_smem(const char* suffix, void** mem, size_t* bytes, size_t min_bytes)
{
    char name[256];
    snprintf(name, sizeof(name), "/%s%s", base_name(), suffix);
    const int fd = shm_open(name, O_RDWR, 0);
    if (fd < 0) {
        report(CUDA_TRANSFER_ERR_SETUP, "Failed to open shared memory '%s': %s", name, strerror(errno));
        return false;
    }
    struct stat st;
    if (fstat(fd, &st) != 0 || (size_t)st.st_size < min_bytes) {
        report(CUDA_TRANSFER_ERR_SETUP, "Shared memory '%s' is smaller than %zu bytes", name, min_bytes);
        close(fd);
        return false;
    }
    void* p = mmap(NULL, (size_t)st.st_size, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    close(fd);
    if (p == MAP_FAILED) {
        report(CUDA_TRANSFER_ERR_SETUP, "Failed to map shared memory '%s': %s", name, strerror(errno));
        return false;
    }
    *mem = p;
    *bytes = (size_t)st.st_size;
    return true;
}

static int open_command_socket(void)
{
    char name[200];
    snprintf(name, sizeof(name), "%s%s", base_name(), COMMAND_SOCKET_SUFFIX);
    const int s = socket(AF_UNIX, SOCK_SEQPACKET | SOCK_CLOEXEC, 0);
    if (s < 0) {
        report(CUDA_TRANSFER_ERR_SETUP, "Failed to create the command socket: %s", strerror(errno));
        return -1;
    }
    struct sockaddr_un addr;
    memset(&addr, 0, sizeof(addr));
    addr.sun_family = AF_UNIX;
    const size_t len = strlen(name);
    memcpy(addr.sun_path + 1, name, len); /* abstract namespace: leading NUL */
    if (connect(s, (struct sockaddr*)&addr, (socklen_t)(offsetof(struct sockaddr_un, sun_path) + 1 + len)) != 0) {
        report(CUDA_TRANSFER_ERR_SETUP, "Failed to connect to the command socket '%s': %s", name, strerror(errno));
        close(s);
        return -1;
    }
    return s;
}

static bool setup_shared_resources(void)
{
    if (!g_data && !open_smem(DATA_SMEM_SUFFIX, &g_data, &g_data_bytes, 1)) goto fail;
    if (!g_params && !open_smem(PARAMETERS_SMEM_SUFFIX, (void**)&g_params, &g_params_bytes, sizeof(SharedMemoryParams)))
        goto fail;
    if (g_sock < 0 && (g_sock = open_command_socket()) < 0) goto fail;
    return true;
fail:
    cleanup_shared_resources();
    return false;
}

static bool send_command(CudaCommand command, size_t data_size)
{
    CommandPipeMessage message;
    memset(&message, 0, sizeof(message));
    message.opcode = command;
    message.data_size = data_size;
    message.frame_count = 0;
    if (send(g_sock, &message, sizeof(message), MSG_NOSIGNAL) != (ssize_t)sizeof(message)) {
        report(CUDA_TRANSFER_ERR_SEND, "Failed to write to the command socket: %s", strerror(errno));
        return false;
    }
    return true;
}

static int64_t now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (int64_t)ts.tv_sec * 1000 + ts.tv_nsec / 1000000;
}

static bool wait_for_response(CommandPipeMessage* message)
{
    const int64_t deadline = now_ms() + g_timeout_ms;
    for (;;) {
        const int64_t left = deadline - now_ms();
        if (left <= 0) {
            report(CUDA_TRANSFER_ERR_TIMEOUT, "Timed out waiting for a response from the command socket after %u ms",
                   g_timeout_ms);
            return false;
        }
        struct pollfd pfd = {g_sock, POLLIN, 0};
        const int r = poll(&pfd, 1, (int)(left > 100 ? 100 : left));
        if (r < 0 && errno != EINTR) {
            report(CUDA_TRANSFER_ERR_PROTOCOL, "poll on the command socket failed: %s", strerror(errno));
            return false;
        }
        if (r <= 0) continue;
        const ssize_t n = recv(g_sock, message, sizeof(*message), 0);
        if (n == 0) {
            report(CUDA_TRANSFER_ERR_DISCONNECTED, "The server closed the command socket");
            return false;
        }
        if (n < 0) {
            if (errno == EINTR || errno == EAGAIN) continue;
            report(CUDA_TRANSFER_ERR_DISCONNECTED, "Failed to read from the command socket: %s", strerror(errno));
            return false;
        }
        if (n != (ssize_t)sizeof(*message)) {
            report(CUDA_TRANSFER_ERR_PROTOCOL, "Invalid message size read from the command socket: %zd", n);
            return false;
        }
        return true;
    }
}

/* send -> ACK -> SUCCESS; returns the announced output size, or -1 (resources released). */
static long long transact(CudaCommand command, size_t data_size)
{
    CommandPipeMessage message;
    if (!send_command(command, data_size)) goto fail;
    if (!wait_for_response(&message)) goto fail;
    if (message.opcode != ACK) {
        if (message.opcode == ERR)
            report(CUDA_TRANSFER_ERR_SERVER, "The server rejected the command");
        else
            report(CUDA_TRANSFER_ERR_PROTOCOL, "Invalid command received from the command socket: %d", (int)message.opcode);
        goto fail;
    }
    if (!wait_for_response(&message)) goto fail;
    if (message.opcode == ERR) {
        report(CUDA_TRANSFER_ERR_SERVER, "Failed to receive valid result from CUDA server");
        goto fail;
    }
    if (message.opcode != SUCCESS) {
        report(CUDA_TRANSFER_ERR_PROTOCOL, "Invalid result received from the command socket: %d", (int)message.opcode);
        goto fail;
    }
    return (long long)message.data_size;
fail:
    cleanup_shared_resources();
    return -1;
}

static bool copy_result(void* dst, long long got, size_t expected, bool exact)
{
    if (got < 0) return false;
    if ((size_t)got > expected || (size_t)got > g_data_bytes || (exact && (size_t)got != expected)) {
        report(CUDA_TRANSFER_ERR_PROTOCOL, "Unexpected result size from server: %lld (expected %zu)", got, expected);
        cleanup_shared_resources();
        return false;
    }
    memcpy(dst, g_data, (size_t)got);
    g_status = CUDA_TRANSFER_OK;
    return true;
}

static void beamform_common(const void* data, size_t data_size, const CudaBeamformerParameters* bp, float* output)
{
    if (!setup_shared_resources()) return;
    if (data_size > g_data_bytes) {
        report(CUDA_TRANSFER_ERR_SIZE, "Data size too large: %zu, Max: %zu", data_size, g_data_bytes);
        return;
    }
    memcpy(&g_params->beamformerParameters, bp, sizeof(CudaBeamformerParameters));
    memcpy(g_data, data, data_size);
    const size_t out = (size_t)bp->output_points[0] * bp->output_points[1] * bp->output_points[2] * 2 * sizeof(float);
    copy_result(output, transact(BEAMFORM_VOLUME, data_size), out, false);
}

void beamform_i16(const short* data, CudaBeamformerParameters bp, float* output)
{
    beamform_common(data, (size_t)bp.rf_raw_dim[0] * bp.rf_raw_dim[1] * sizeof(short), &bp, output);
}

void beamform_f32(const float* data, CudaBeamformerParameters bp, float* output)
{
    beamform_common(data, (size_t)bp.rf_raw_dim[0] * bp.rf_raw_dim[1] * sizeof(float), &bp, output);
}

void motion_detect_f32(const float* images, NCCMotionParameters params, float* motion_maps)
{
    const size_t data_size = (size_t)params.image_dims[0] * params.image_dims[1] * params.frame_count * sizeof(float);
    if (!setup_shared_resources()) return;
    if (data_size > g_data_bytes) {
        report(CUDA_TRANSFER_ERR_SIZE, "Data size too large: %zu, Max: %zu", data_size, g_data_bytes);
        return;
    }
    memcpy(&g_params->nccMotionParameters, &params, sizeof(NCCMotionParameters));
    memcpy(g_data, images, data_size);
    const size_t out = (size_t)params.motion_grid_dims[0] * params.motion_grid_dims[1] * 4 * sizeof(float) *
                       params.frame_count;
    copy_result(motion_maps, transact(NCC_MOTION_DETECT, data_size), out, false);
}

void corr_images_f32(const float* template_image, const float* source_image, CorrImagesParameters params,
                     float* corr_map)
{
    if (params.template_dims[0] == 0 || params.template_dims[1] == 0 || params.source_dims[0] == 0 ||
        params.source_dims[1] == 0) {
        report(CUDA_TRANSFER_ERR_SIZE, "Invalid corr_images dimensions");
        return;
    }
    if (params.template_dims[0] > params.source_dims[0] || params.template_dims[1] > params.source_dims[1]) {
        report(CUDA_TRANSFER_ERR_SIZE, "Template dimensions must be <= source dimensions");
        return;
    }
    const size_t tpl = (size_t)params.template_dims[0] * params.template_dims[1] * sizeof(float);
    const size_t src = (size_t)params.source_dims[0] * params.source_dims[1] * sizeof(float);
    const size_t out = ((size_t)params.source_dims[0] - params.template_dims[0] + 1) *
                       ((size_t)params.source_dims[1] - params.template_dims[1] + 1) * sizeof(float);
    if (!setup_shared_resources()) return;
    if (tpl + src > g_data_bytes) {
        report(CUDA_TRANSFER_ERR_SIZE, "Data size too large: %zu, Max: %zu", tpl + src, g_data_bytes);
        return;
    }
    memcpy(&g_params->corrImagesParameters, &params, sizeof(CorrImagesParameters));
    memcpy(g_data, template_image, tpl);
    memcpy((char*)g_data + tpl, source_image, src);
    copy_result(corr_map, transact(CORR_IMAGES, tpl + src), out, true);
}

void deinit(void) { cleanup_shared_resources(); }

int cuda_transfer_status(void) { return g_status; }

void cuda_transfer_set_timeout_ms(unsigned int ms) { g_timeout_ms = ms ? ms : RESPONSE_POLL_TIMEOUT_MS; }
