/*
 * Client side of the out-of-process transfer path: the functions of upstream's client library
 * (test_app/client_lib/cuda_transfer.h:16-27, cuda_transfer.c:370-467) with the same names and
 * arguments, built as libcuda_transfer.so (plain C, no CUDA). Each call places the parameters and
 * the input in the server's shared memory, sends one command over the command socket, waits for
 * ACK and then for the result, and copies the output back. Errors are printed on stderr as
 * upstream does; cuda_transfer_status() also returns a code for the last call.
 *
 * The server is cutb_transfer_server (or cutb_server_serve in libcuda_toolkit_b200.so).
 */
#ifndef CUDA_TRANSFER_H
#define CUDA_TRANSFER_H

#ifdef __cplusplus
extern "C" {
#endif

#include "communication_params.h"

#ifndef LIB_FN
#if defined(_WIN32)
#define LIB_FN __declspec(dllexport)
#else
#define LIB_FN __attribute__((visibility("default")))
#endif
#endif

LIB_FN void beamform_i16(const short* data, CudaBeamformerParameters bp, float* output);

LIB_FN void beamform_f32(const float* data, CudaBeamformerParameters bp, float* output);

LIB_FN void motion_detect_f32(const float* images, NCCMotionParameters params, float* motion_maps);

LIB_FN void corr_images_f32(const float* template_image, const float* source_image, CorrImagesParameters params,
                            float* corr_map);

/* Unmaps the shared memory and closes the command socket. */
LIB_FN void deinit(void);

/* Not upstream: result of the last call and the response timeout (upstream: 20 minutes). */
enum {
    CUDA_TRANSFER_OK = 0,
    CUDA_TRANSFER_ERR_SETUP = 1,        /* shared memory or command socket unavailable */
    CUDA_TRANSFER_ERR_SIZE = 2,         /* input or output does not fit, or invalid dimensions */
    CUDA_TRANSFER_ERR_SEND = 3,         /* the command could not be sent */
    CUDA_TRANSFER_ERR_TIMEOUT = 4,      /* no response within the timeout */
    CUDA_TRANSFER_ERR_PROTOCOL = 5,     /* unexpected message */
    CUDA_TRANSFER_ERR_SERVER = 6,       /* the server answered ERR */
    CUDA_TRANSFER_ERR_DISCONNECTED = 7, /* the server closed the connection */
};
LIB_FN int cuda_transfer_status(void);
LIB_FN void cuda_transfer_set_timeout_ms(unsigned int ms);

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* CUDA_TRANSFER_H */
