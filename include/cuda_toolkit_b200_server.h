/*
 * Server side of the out-of-process transfer path (upstream test_app/src/transfer_server.cpp:
 * 8-258 and TestApp::_message_loop / _handle_*_command, test_app.cpp:42-304), over the POSIX
 * command socket and shared-memory segments described in communication_params.h.
 *
 * The built-in handlers call this library's cuda_toolkit::beamform, ::motion_detection and
 * ::corr_images on the shared data segment, which is page-locked for the device copies on the
 * first such command. Results go through a server-owned staging buffer and reach the segment
 * only while the requesting client is still connected. A handler installed with cutb_server_set_handler replaces them (it runs
 * on the serving thread, after the server has answered ACK).
 *
 * The executable cutb_transfer_server wraps these calls.
 */
#ifndef CUDA_TOOLKIT_B200_SERVER_H
#define CUDA_TOOLKIT_B200_SERVER_H

#include <stdint.h>

#include "communication_params.h"
#include "cuda_toolkit_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cutb_server cutb_server;

/* Replacement request handler: reads the request (params, data[0, data_bytes)), writes at most
 * out_capacity bytes at `out` (a server-owned buffer, copied to the start of the data segment
 * while the client still waits) and sets *out_bytes. Returns 0 for SUCCESS, anything else for
 * ERR. */
typedef int (*cutb_server_handler)(int opcode, const SharedMemoryParams* params, const uint8_t* data,
                                   uint64_t data_bytes, uint8_t* out, uint64_t out_capacity, uint64_t* out_bytes,
                                   void* user);

/* Creates the command socket "<name>_command" and the segments "/<name>_data" (data_bytes;
 * 0 = DATA_SMEM_SIZE) and "/<name>_parameters". name NULL = $CUDA_TRANSFER_NAME or "cuda".
 * Segments of the same name left by a previous server are replaced. */
CUTB_API cutb_server* cutb_server_create(const char* name, uint64_t data_bytes);
CUTB_API void cutb_server_set_handler(cutb_server* server, cutb_server_handler handler, void* user);

/* Serves commands until max_commands (> 0) have been handled, no command arrived for
 * idle_timeout_ms (> 0; upstream: one hour), or cutb_server_stop was called. Returns the number
 * of commands handled, -1 on a socket error. One client at a time; a client that disconnects is
 * replaced by the next one. */
CUTB_API int cutb_server_serve(cutb_server* server, int max_commands, int idle_timeout_ms);

/* Makes a running (or the next) cutb_server_serve return within ~100 ms; callable from any
 * thread. */
CUTB_API void cutb_server_stop(cutb_server* server);

/* Closes the socket and removes the segments. */
CUTB_API void cutb_server_destroy(cutb_server* server);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_TOOLKIT_B200_SERVER_H */
