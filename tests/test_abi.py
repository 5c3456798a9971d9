"""The drop-in boundary: struct layout, exported symbols, host-only entry points (no GPU)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from cuda_ultrasound_toolkit_b200.params import CudaBeamformerParameters

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")

# Offsets of the upstream struct on x86-64 (cuda_beamformer_parameters.h:109-172).
OFFSETS = {
    "xdc_transform": 0, "xdc_element_pitch": 64, "rf_raw_dim": 72, "dec_data_dim": 88, "decode": 104,
    "das_shader_id": 108, "time_offset": 112, "output_points": 116, "output_min_coordinate": 132,
    "output_max_coordinate": 148, "sampling_frequency": 164, "center_frequency": 168, "speed_of_sound": 172,
    "fn_tx": 184, "fn_rx": 188, "interpolate": 192, "coherency_weighting": 196, "channel_mapping": 200,
    "sparse_elements": 712, "foci": 1224, "tx_orientation": 4296, "rx_orientation": 4300,
    "readi_group_count": 4304, "readi_group_id": 4308, "filter_length": 4832, "rf_filter": 4836,
    "data_type": 8932, "apo_type": 8936, "to_power": 8940, "sample_type": 8944,
}


def test_ctypes_struct_layout():
    assert ctypes.sizeof(CudaBeamformerParameters) == 8948
    for name, off in OFFSETS.items():
        assert getattr(CudaBeamformerParameters, name).offset == off, name


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_header_layout_compiles(tmp_path, lang):
    """The public header compiles as C and C++ and has the upstream layout."""
    src = tmp_path / ("t.c" if lang == "c" else "t.cpp")
    checks = "\n".join(
        f'_Static_assert(offsetof(CudaBeamformerParameters, {k}) == {v}, "{k}");' if lang == "c" else
        f'static_assert(offsetof(CudaBeamformerParameters, {k}) == {v}, "{k}");' for k, v in OFFSETS.items())
    src.write_text(
        '#include <stddef.h>\n#include "cuda_beamformer_parameters.h"\n#include "cuda_toolkit_ogl.h"\n'
        '#include "cuda_toolkit_matlab.h"\n#include "cuda_toolkit_b200.h"\n'
        + ('#include "cuda_toolkit.hpp"\n' if lang == "c++" else "") + checks +
        "\nint main(void) { return (int)sizeof(CudaBeamformerParameters) - 8948; }\n")
    exe = tmp_path / "t"
    cc = ["gcc", "-std=c11"] if lang == "c" else ["g++", "-std=c++20"]
    subprocess.run(cc + ["-I", INCLUDE, str(src), "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)]).returncode == 0


def test_motion_parameter_layout(tmp_path):
    """NccMotionParameters / CorrImagesParameters: the ctypes mirrors match the C header."""
    from cuda_ultrasound_toolkit_b200.params import CorrImagesParameters, NccMotionParameters
    fields = [f[0] for f in NccMotionParameters._fields_]
    src = tmp_path / "m.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "cuda_beamformer_parameters.h"\n'
                   "int main(void) {\n"
                   + "".join(f'printf("%zu\\n", offsetof(NCCMotionParameters, {f}));\n' for f in fields)
                   + 'printf("%zu\\n%zu\\n", sizeof(NCCMotionParameters), sizeof(CorrImagesParameters));\n'
                   "return 0; }\n")
    exe = tmp_path / "m"
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals[:-2] == [getattr(NccMotionParameters, f).offset for f in fields]
    assert vals[-2:] == [ctypes.sizeof(NccMotionParameters), ctypes.sizeof(CorrImagesParameters)]


def test_plan_options_layout(tmp_path):
    """cutb_options: the ctypes mirror the Python layer passes to cutb_plan_create matches the C
    header (every named field's offset and the struct size)."""
    from cuda_ultrasound_toolkit_b200.api import _Options
    fields = [f[0] for f in _Options._fields_ if f[0] != "reserved"]
    src = tmp_path / "o.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "cuda_toolkit_b200.h"\n'
                   "int main(void) {\n"
                   + "".join(f'printf("%zu\\n", offsetof(cutb_options, {f}));\n' for f in fields)
                   + 'printf("%zu\\n", sizeof(cutb_options));\n'
                   "return 0; }\n")
    exe = tmp_path / "o"
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals[:-1] == [getattr(_Options, f).offset for f in fields]
    assert vals[-1] == ctypes.sizeof(_Options) == 64


def _declared_functions(only=None, skip=("cuda_transfer.h",)):
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h") or (only and fn != only) or (not only and fn in skip):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"(?:EXPORT_FN|LIB_FN|CUTB_API)\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(native):
    declared = _declared_functions()
    assert {"init_cuda_configuration", "cuda_decode", "cuda_hilbert", "beamform_i16_matlab",
            "cutb_plan_create", "cuda_register_device_buffer"} <= declared
    for name in declared:
        assert hasattr(native, name), name
    # cuda_toolkit::beamform / motion_detection / corr_images (C++ linkage, cuda_toolkit.hpp)
    out = subprocess.run(["nm", "-DC", "--defined-only", native._name], capture_output=True, text=True).stdout
    for sym in ("cuda_toolkit::beamform(", "cuda_toolkit::motion_detection(", "cuda_toolkit::corr_images("):
        assert sym in out, sym


def test_transfer_client_exports_every_declared_symbol(native):
    """cuda_transfer.h (the drop-in of upstream's client library) is implemented by
    libcuda_transfer.so, a plain C library with no CUDA dependency."""
    from cuda_ultrasound_toolkit_b200 import transfer
    declared = _declared_functions(only="cuda_transfer.h")
    assert {"beamform_i16", "beamform_f32", "motion_detect_f32", "corr_images_f32", "deinit"} <= declared
    client = transfer.client()
    for name in declared:
        assert hasattr(client, name), name
    out = subprocess.run(["ldd", transfer.CLIENT_PATH], capture_output=True, text=True).stdout
    assert "cuda" not in out.replace("libcuda_transfer", "")


def test_library_links_no_fft_or_blas(native):
    """No cuFFT / cuBLAS / NPP: every kernel on the path is this library's own."""
    out = subprocess.run(["ldd", native._name], capture_output=True, text=True).stdout
    for bad in ("cufft", "cublas", "npp", "oracle"):
        assert bad not in out


def test_encoding_matrix_host_entry_point(native, orc):
    from cuda_ultrasound_toolkit_b200 import encoding_matrix
    for n in (1, 2, 8, 12, 20, 24, 40, 64, 96, 128, 160, 256, 320, 384, 512, 640, 768, 1024):
        for ordering in (1, 2):
            h = encoding_matrix(n, ordering)
            assert (h.astype(np.int64) @ h.T.astype(np.int64) == n * np.eye(n, dtype=np.int64)).all()
            assert (h == orc.encoding_matrix(n, ordering)).all(), (n, ordering)


def test_encoding_matrix_rejects_unsupported_orders(native):
    from cuda_ultrasound_toolkit_b200 import CutbError, encoding_matrix
    for n in (0, 3, 6, 36, 60, 1025, 2048):
        with pytest.raises(CutbError) as e:
            encoding_matrix(n, 1)
        assert e.value.code == 2  # CUTB_ERR_UNSUPPORTED
