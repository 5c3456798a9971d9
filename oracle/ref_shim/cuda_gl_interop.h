/* Stand-in for CUDA's cuda_gl_interop.h when the upstream sources are compiled for the CPU
 * (test infrastructure only): declares the few GL-interop calls upstream makes, without any
 * OpenGL header. The emulation layer (oracle/ref_shim/shim.cpp) resolves buffer ids through
 * a registry of host buffers. */
#pragma once
#include <cuda_runtime_api.h>
typedef unsigned int GLuint;
typedef unsigned int GLenum;
extern "C" {
cudaError_t cudaGraphicsGLRegisterBuffer(cudaGraphicsResource_t* resource, GLuint buffer, unsigned int flags);
}
