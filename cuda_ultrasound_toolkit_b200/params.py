"""ctypes mirror of CudaBeamformerParameters and its enums.

Field order, types and offsets follow include/cuda_beamformer_parameters.h, which is
layout-identical to the upstream cuda_toolkit/src/public/cuda_beamformer_parameters.h:15-172
(x86-64: sizeof == 8948 bytes). The MATLAB mirror of the same struct is upstream
cuda_toolkit/src/public/matlab/CudaBeamformerParameters.m.
"""
import ctypes
import enum

MAX_ACQ_COUNT = 256
MAX_CHANNEL_COUNT = 256
MAX_FILTER_LENGTH = 1024


class RCAOrientation(enum.IntEnum):
    ORIENT_NONE = 0
    ORIENT_ROWS = 1
    ORIENT_COLS = 2


class SampleType(enum.IntEnum):
    SAMPLE_NORMAL = 0
    SAMPLE_BANDPASS = 1


class SequenceId(enum.IntEnum):
    FORCES = 0
    UFORCES = 1
    HERCULES = 2
    RCA_VLS = 3
    RCA_TPW = 4
    UHURCULES = 5
    RACES = 6
    EPIC_FORCES = 7
    EPIC_UFORCES = 8
    EPIC_UHERCULES = 9
    FLASH = 10
    HERO_PA = 11
    MIXES_S = 100


class InputDataTypes(enum.IntEnum):
    INVALID_TYPE = 0
    TYPE_I16 = 1
    TYPE_F32 = 2
    TYPE_F32C = 3
    TYPE_U8 = 4


class EncodingMatrix(enum.IntEnum):
    NONE = 0
    HADAMARD = 1
    WALSH = 2


class ApoType(enum.IntEnum):
    RX_HANN = 0
    RX_TO_SIN = 1
    TX_TO_SIN = 2
    BOTH_TO_SIN = 3


_u = ctypes.c_uint
_f = ctypes.c_float
_i = ctypes.c_int


class CudaBeamformerParameters(ctypes.Structure):
    _fields_ = [
        ("xdc_transform", _f * 16),
        ("xdc_element_pitch", _f * 2),
        ("rf_raw_dim", _u * 4),
        ("dec_data_dim", _u * 4),
        ("decode", _i),
        ("das_shader_id", _i),
        ("time_offset", _f),
        ("output_points", _u * 4),
        ("output_min_coordinate", _f * 4),
        ("output_max_coordinate", _f * 4),
        ("sampling_frequency", _f),
        ("center_frequency", _f),
        ("speed_of_sound", _f),
        ("off_axis_pos", _f),
        ("beamform_plane", _i),
        ("fn_tx", _f),
        ("fn_rx", _f),
        ("interpolate", ctypes.c_bool),
        ("coherency_weighting", _f),
        ("channel_mapping", ctypes.c_short * MAX_CHANNEL_COUNT),
        ("sparse_elements", ctypes.c_short * MAX_CHANNEL_COUNT),
        ("foci", _f * (MAX_ACQ_COUNT * 3)),
        ("tx_orientation", _i),
        ("rx_orientation", _i),
        ("readi_group_count", _u),
        ("readi_group_id", _u),
        ("mixes_count", _u),
        ("mixes_offset", _u),
        ("mixes_rows", _u * 128),
        ("filter_length", _u),
        ("rf_filter", _f * MAX_FILTER_LENGTH),
        ("data_type", _i),
        ("apo_type", _i),
        ("to_power", _i),
        ("sample_type", _i),
    ]

    def copy(self):
        other = CudaBeamformerParameters()
        ctypes.memmove(ctypes.byref(other), ctypes.byref(self), ctypes.sizeof(self))
        return other

    @property
    def dims(self):
        """(S, C, T) = samples, receive channels, transmits."""
        return tuple(int(v) for v in self.dec_data_dim[:3])

    @property
    def volume_shape(self):
        """(Z, Y, X) of the complex output volume."""
        x, y, z = (int(v) for v in self.output_points[:3])
        return (z, y, x)


assert ctypes.sizeof(CudaBeamformerParameters) == 8948


class NccMotionParameters(ctypes.Structure):
    """Block-matching parameters (cuda_beamformer_parameters.h:91-107 upstream). Index 0 of every
    pair is the fastest image axis (x, the image width), index 1 the slow axis (y)."""

    _fields_ = [
        ("patch_size", _u),
        ("motion_grid_spacing", _u),
        ("motion_grid_dims", _u * 2),
        ("scale_dims", _u * 2),
        ("search_margins", _u * 2),
        ("abs_cor_threshold", _f),
        ("rel_cor_threshold", _f),
        ("min_patch_variance", _f),
        ("use_subpixel", ctypes.c_bool),
        ("reference_frame", _u),
        ("neighbour_compare", ctypes.c_bool),
        ("frame_count", _u),
        ("image_dims", _u * 2),
        ("data_type", _i),
    ]

    FIELDS = ("patch_size", "motion_grid_spacing", "abs_cor_threshold", "rel_cor_threshold",
              "min_patch_variance", "use_subpixel", "reference_frame", "neighbour_compare", "frame_count")
    PAIRS = ("motion_grid_dims", "scale_dims", "search_margins", "image_dims")

    @classmethod
    def make(cls, **kw):
        p = cls()
        p.data_type = InputDataTypes.TYPE_F32
        for k, v in kw.items():
            if k in cls.PAIRS:
                getattr(p, k)[0], getattr(p, k)[1] = int(v[0]), int(v[1])
            else:
                setattr(p, k, v)
        return p

    def as_dict(self):
        d = {k: getattr(self, k) for k in self.FIELDS}
        d.update({k: tuple(getattr(self, k)) for k in self.PAIRS})
        return d


class CorrImagesParameters(ctypes.Structure):
    """Image sizes of corr_images_f32_matlab, index 0 = width (fastest axis)."""

    _fields_ = [("template_dims", _u * 2), ("source_dims", _u * 2)]


assert ctypes.sizeof(NccMotionParameters) == 72
