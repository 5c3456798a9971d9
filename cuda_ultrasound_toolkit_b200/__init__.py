"""B200-native RF -> volume pipeline (convert + reorder + Hadamard decode, match-filtered
Hilbert analytic signal, 3-D delay-and-sum), a drop-in for the cuda_toolkit::beamform and
GL-buffer C ABI of the upstream cuda_ultrasound_toolkit.

The compute path is the native library libcuda_toolkit_b200.so (hand-written sm_100a
kernels); this package is its Python host mirror. There is no CPU fallback.
"""
from .params import (ApoType, CudaBeamformerParameters, EncodingMatrix, InputDataTypes, RCAOrientation,
                     SampleType, SequenceId)
from .api import (Batch, CutbError, Plan, RfSession, beamform, beamform_f32, beamform_i16, encoding_matrix, last_error,
                  lib, library_path)

__all__ = [
    "ApoType", "CudaBeamformerParameters", "EncodingMatrix", "InputDataTypes", "RCAOrientation", "SampleType",
    "SequenceId", "Batch", "CutbError", "Plan", "RfSession", "beamform", "beamform_f32", "beamform_i16", "encoding_matrix",
    "last_error", "lib", "library_path",
]
