/*
 * Parameter block shared by every entry point of the RF -> volume library.
 *
 * This header is a drop-in replacement for the upstream toolkit's
 * cuda_toolkit/src/public/cuda_beamformer_parameters.h:15-172. The struct and
 * enum layout must stay byte-identical to it, because callers (MATLAB mirror
 * classes, the OpenGL host app, the IPC harness) build the struct themselves
 * and pass it by value or by reference. Field names, types and order are
 * therefore fixed; the x86-64 layout is pinned below with static_asserts
 * (sizeof == 8948 bytes).
 *
 * Which fields the hot path honours is documented beside each field.
 */
#ifndef CUDA_BEAMFORMER_PARAMETERS_H
#define CUDA_BEAMFORMER_PARAMETERS_H

#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Compile-time capacity of the fixed-size arrays inside the struct. */
#define MAX_ACQ_COUNT 256
#define MAX_CHANNEL_COUNT 256
#define MAX_FILTER_LENGTH 1024

typedef unsigned int uint;

/* Row-column array orientation of the transmit or receive aperture. */
typedef enum RCAOrientation {
    ORIENT_NONE = 0,
    ORIENT_ROWS = 1,
    ORIENT_COLS = 2,
} RCAOrientation;

/* NORMAL = real RF sampled at fs; BANDPASS = interleaved IQ pairs (not on the hot path). */
typedef enum SampleType {
    SAMPLE_NORMAL = 0,
    SAMPLE_BANDPASS = 1,
} SampleType;

/* Transmit orientation in the high nibble, receive orientation in the low nibble. */
typedef enum {
    INVALID = 0,
    NO_TX_ROW_RX = 1,
    NO_TX_COL_RX = 2,
    ROW_TX_ROW_RX = 17,
    ROW_TX_COL_RX = 18,
    COL_TX_ROW_RX = 33,
    COL_TX_COL_RX = 34,
} PackedTROrientation;

/* Carried in the struct for layout compatibility; the hot path ignores it. */
typedef enum BeamformPlane {
    PLANE_XZ = 0,
    PLANE_YZ = 1,
    PLANE_XY = 2,
    PLANE_ARBITRARY = 3,
} BeamformPlane;

/* Acquisition sequence; selects the delay model of the delay-and-sum stage. */
typedef enum SequenceId {
    FORCES = 0,
    UFORCES = 1,
    HERCULES = 2,
    RCA_VLS = 3,
    RCA_TPW = 4,
    UHURCULES = 5,
    RACES = 6,
    EPIC_FORCES = 7,
    EPIC_UFORCES = 8,
    EPIC_UHERCULES = 9,
    FLASH = 10,
    HERO_PA = 11,
    MIXES_S = 100,
} SequenceId;

/* Element type of the raw RF buffer. Only I16 and F32 are accepted. */
typedef enum InputDataTypes {
    INVALID_TYPE = 0,
    TYPE_I16 = 1,
    TYPE_F32 = 2,
    TYPE_F32C = 3,
    TYPE_U8 = 4,
} InputDataTypes;

/* Transmit encoding: none (plain reorder), Hadamard, or Walsh (sequency-ordered Hadamard). */
typedef enum EncodingMatrix {
    NONE = 0,
    HADAMARD = 1,
    WALSH = 2,
} EncodingMatrix;

/* Apodization model used by the delay-and-sum stage. */
typedef enum ApoType {
    RX_HANN = 0,
    RX_TO_SIN = 1,
    TX_TO_SIN = 2,
    BOTH_TO_SIN = 3,
} ApoType;

/* Parameters of the (out-of-scope) NCC motion detection entry points; layout only. */
typedef struct NccMotionParameters {
    uint patch_size;
    uint motion_grid_spacing;
    uint motion_grid_dims[2];
    uint scale_dims[2];
    uint search_margins[2];
    float abs_cor_threshold;
    float rel_cor_threshold;
    float min_patch_variance;
    bool use_subpixel;
    uint reference_frame;
    bool neighbour_compare;
    uint frame_count;
    uint image_dims[2];
    InputDataTypes data_type;
} NCCMotionParameters;

typedef struct CudaBeamformerParameters {
    /* Transducer and sequence description. */
    float xdc_transform[16];      /* 4x4 column-major; only [12], [13] (half aperture x, y) are read */
    float xdc_element_pitch[2];   /* [m] element pitch {x (columns), y (rows)} */

    uint rf_raw_dim[4];           /* [samples*transmits + padding, raw channels]; [2], [3] ignored */
    uint dec_data_dim[4];         /* [samples S, receive channels C, transmits T]; [3] ignored */

    EncodingMatrix decode;        /* NONE = reorder only */
    SequenceId das_shader_id;     /* HERCULES / FORCES on the hot path */
    float time_offset;            /* [s] delay correction; truncated to whole samples */

    /* Output grid. */
    uint output_points[4];        /* [X, Y, Z, frames]; frames ignored */
    float output_min_coordinate[4];
    float output_max_coordinate[4];

    float sampling_frequency;     /* [Hz] */
    float center_frequency;       /* [Hz] */
    float speed_of_sound;         /* [m/s] */

    float off_axis_pos;           /* ignored */
    BeamformPlane beamform_plane; /* ignored */

    float fn_tx;                  /* transmit f-number (FORCES Hann apodization) */
    float fn_rx;                  /* receive f-number (Hann apodization); 0 = uniform */
    bool interpolate;             /* false = linear, true = cubic (Catmull-Rom) */
    float coherency_weighting;    /* coherence-factor exponent, clamped to [0, 1]; 0 = off */

    /* Large tables. */
    short channel_mapping[MAX_CHANNEL_COUNT]; /* raw channel feeding each receive channel */
    short sparse_elements[MAX_CHANNEL_COUNT]; /* UFORCES virtual sources */
    float foci[MAX_ACQ_COUNT * 3];            /* per-transmit focus; only foci[0..2] on the hot path */

    RCAOrientation tx_orientation;
    RCAOrientation rx_orientation;

    /* READI sub-aperture encoding. */
    uint readi_group_count;       /* 0 or 1 = no READI */
    uint readi_group_id;

    uint mixes_count;             /* ignored */
    uint mixes_offset;            /* ignored */
    uint mixes_rows[128];         /* ignored */

    uint filter_length;           /* match filter taps; 0 = no filter */
    float rf_filter[MAX_FILTER_LENGTH];

    InputDataTypes data_type;     /* TYPE_I16 or TYPE_F32 */
    ApoType apo_type;
    int to_power;                 /* exponent of the sine apodization */

    SampleType sample_type;       /* only SAMPLE_NORMAL runs the RF front end */
} CudaBeamformerParameters;

/* Parameters of the (out-of-scope) image correlation entry points; layout only. */
typedef struct CorrImagesParameters {
    unsigned int template_dims[2];
    unsigned int source_dims[2];
} CorrImagesParameters;

#ifdef __cplusplus
}
#endif

#if defined(__cplusplus) && defined(__x86_64__)
#include <cstddef>
static_assert(sizeof(CudaBeamformerParameters) == 8948, "ABI: CudaBeamformerParameters size");
static_assert(offsetof(CudaBeamformerParameters, rf_raw_dim) == 72, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, decode) == 104, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, output_points) == 116, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, sampling_frequency) == 164, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, fn_tx) == 184, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, interpolate) == 192, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, coherency_weighting) == 196, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, channel_mapping) == 200, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, foci) == 1224, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, tx_orientation) == 4296, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, readi_group_count) == 4304, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, filter_length) == 4832, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, rf_filter) == 4836, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, data_type) == 8932, "ABI offset");
static_assert(offsetof(CudaBeamformerParameters, sample_type) == 8944, "ABI offset");
#endif

#endif /* CUDA_BEAMFORMER_PARAMETERS_H */
