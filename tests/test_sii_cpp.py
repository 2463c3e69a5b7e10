"""The main path's C++ entry points with the reference's own types and linkage
(include/svdimager_b200_sii.hpp; SVDIntegratedImager.cu:39-86): a caller written against those
declarations (tests/sii_caller/main.cpp, the way the reference's main uses them) compiles and links
against the library unchanged, and on the GPU its image equals the engine's and the oracle's."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "svdimager_b200", "lib")
# the reference's mangled names: int FIpipeDevice(const DevicePreprocessBuffers&, float*, size_t, float),
# void preprocess_measurement_set_gpu(const HostMeasurementSetData&, DevicePreprocessBuffers&),
# void free_device_preprocess_buffers(DevicePreprocessBuffers&)
SII_SYMBOLS = ("_Z12FIpipeDeviceRK23DevicePreprocessBuffersPfmf",
               "_Z30preprocess_measurement_set_gpuRK22HostMeasurementSetDataR23DevicePreprocessBuffers",
               "_Z30free_device_preprocess_buffersR23DevicePreprocessBuffers")


def _build_caller(tmp_path):
    exe = str(tmp_path / "sii_caller")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", exe,
                           os.path.join(ROOT, "tests", "sii_caller", "main.cpp"), "-L", LIB_DIR,
                           "-lsvdimager_b200", f"-Wl,-rpath,{LIB_DIR}"])
    return exe


def test_library_exports_the_reference_main_path_symbols():
    from svdimager_b200 import api
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH], capture_output=True, text=True).stdout
    for sym in SII_SYMBOLS:
        assert sym in out, sym


def test_caller_against_reference_declarations_links(tmp_path):
    assert os.path.exists(_build_caller(tmp_path))


def _write_snapshot(path, s, N, cell):
    with open(path, "wb") as f:
        np.array([s.num_rows, s.num_channels, N], np.uint64).tofile(f)
        np.array([cell, s.array_center_x], np.float32).tofile(f)
        for a in (s.uvw, s.frequencies_hz, s.vis0_real, s.vis0_imag, s.vis3_real, s.vis3_imag):
            np.ascontiguousarray(a, np.float32).tofile(f)
        for a in (s.flag0, s.flag3):
            np.ascontiguousarray(a, np.uint8).tofile(f)
        for a in (s.weight0, s.weight3):
            np.ascontiguousarray(a, np.float32).tofile(f)


@pytest.mark.gpu
def test_caller_image_equals_engine_and_oracle(cuda_device, small_snapshot, tmp_path):
    from oracle import oracle as O
    from svdimager_b200 import api
    s = small_snapshot
    N, cell = s.image_size, s.cell_size
    exe = _build_caller(tmp_path)
    _write_snapshot(tmp_path / "snap.bin", s, N, cell)
    r = subprocess.run([exe, str(tmp_path / "snap.bin"), str(tmp_path / "img.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    img = np.fromfile(tmp_path / "img.bin", np.float32).reshape(N, N)
    with api.Engine() as e:
        ref = e.image(s)
    assert O.rel_rms(img, ref) < 1e-6
    assert O.rel_rms(img, O.image_sii(s).image) < 1e-5
