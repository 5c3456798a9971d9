/*
 * Wire format of the out-of-process transfer path (upstream test_app/src/communication_params.h:
 * 10-59), carried over POSIX primitives instead of Win32 ones:
 *
 *   upstream (Windows)                      here (Linux)
 *   named pipe \\.\pipe\cuda_command         SOCK_SEQPACKET Unix socket (abstract name
 *     (message mode, one instance)             "cuda_command"), one client at a time
 *   file mapping Local\cuda_data (2 GB)      POSIX shm "/cuda_data" (size chosen by the server)
 *   file mapping Local\cuda_parameters       POSIX shm "/cuda_parameters" (SharedMemoryParams)
 *
 * The messages and the shared parameter block keep upstream's C layout (x86-64), so a client
 * built against upstream's header speaks the same bytes. Exchange: the client writes the
 * parameter block and the input into shared memory and sends {opcode, data_size}; the server
 * answers ACK (or ERR when the request is invalid), runs the request, writes the output at the
 * start of the data segment and answers SUCCESS with the output size in data_size (or ERR).
 *
 * The base name ("cuda") can be changed with the environment variable CUDA_TRANSFER_NAME on
 * both sides: the socket is then "<name>_command" and the segments "/<name>_data" and
 * "/<name>_parameters".
 */
#ifndef COMMUNICATION_PARAMS_H
#define COMMUNICATION_PARAMS_H

#ifdef __cplusplus
extern "C" {
#endif

#include "cuda_beamformer_parameters.h"

#define CUDA_TRANSFER_DEFAULT_NAME "cuda"
#define COMMAND_SOCKET_SUFFIX "_command"
#define DATA_SMEM_SUFFIX "_data"
#define PARAMETERS_SMEM_SUFFIX "_parameters"

#define MEGABYTE (1024U * 1024U)
#define GIGABYTE (1024U * 1024U * 1024U)

#define DATA_SMEM_SIZE 0x80000000UL /* default data segment: 2 GB */

/* What the client asks for (and the server's answers). */
typedef enum CudaCommand {
    ERR = 0,
    ACK = 1,
    SUCCESS = 2,
    BEAMFORM_VOLUME = 3,
    SVD_FILTER = 4,
    NCC_MOTION_DETECT = 5,
    CORR_IMAGES = 6,
} CudaCommand;

typedef struct CommandPipeMessage {
    CudaCommand opcode;
    unsigned long long data_size; /* request: input bytes; SUCCESS: output bytes */
    int frame_count;
} CommandPipeMessage;

typedef struct SVDParameters {
    int frame_count;
    int filter_indicies[256]; /* singular values to remove (upstream has no server-side handler) */
} SVDParameters;

typedef struct SharedMemoryParams {
    CudaBeamformerParameters beamformerParameters;
    SVDParameters svdParameters;
    NCCMotionParameters nccMotionParameters;
    CorrImagesParameters corrImagesParameters;
} SharedMemoryParams;

#if defined(__x86_64__) && !defined(__cplusplus)
_Static_assert(sizeof(CommandPipeMessage) == 24, "CommandPipeMessage layout");
#elif defined(__x86_64__)
static_assert(sizeof(CommandPipeMessage) == 24, "CommandPipeMessage layout");
#endif

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* COMMUNICATION_PARAMS_H */
