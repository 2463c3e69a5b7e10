"""The C-ABI library loads on a machine without a GPU and exports every function the public header
declares; host-side helpers (FITS, bundle, CLI argument handling) behave like the reference's."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "svdimager_b200.h")


def test_library_loads_and_exports_header_functions():
    from svdimager_b200 import api
    L = api.lib()
    text = open(HEADER).read()
    declared = set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(svdi_\w+)\s*\(", text, re.M))
    declared.discard("svdi_options")
    assert declared, "no declarations parsed"
    assert declared <= set(api.EXPORTED_SYMBOLS), declared - set(api.EXPORTED_SYMBOLS)
    for name in api.EXPORTED_SYMBOLS:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH], capture_output=True, text=True).stdout
    # C++-linkage archive entry with the reference's exact signature (pipe_interface.cpp:8)
    assert "_Z6FIpipePfS_S_S_S_mmf" in out


def test_struct_sizes_match_c_layout():
    from svdimager_b200 import api
    import ctypes
    assert ctypes.sizeof(api.HostMS) == 8 * 13 + 8  # 13 size_t/pointers + float (padded)
    o = api.default_options()
    assert o.k_rule == api.KRULE_BUCKET and o.support == 8 and abs(o.beta - 15.3704324328) < 1e-12
    assert o.sigma == 1.5 and o.edge_mode == api.EDGE_CLIP and o.coord_mode == api.COORD_FP64


def test_error_reporting_without_gpu():
    from svdimager_b200 import api
    with pytest.raises(api.SvdiError) as ei:
        api.FIpipe(np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32),
                   np.eye(3, dtype=np.float32), 16, 1e-3)
    assert ei.value.status == 2  # SVDI_ERR_EMPTY_INPUT
    with pytest.raises(api.SvdiError) as ei:
        api.FIpipe(np.ones(4, np.float32), np.ones(4, np.float32), np.ones(12, np.float32),
                   np.eye(3, dtype=np.float32), 16, -1.0)
    assert ei.value.status == 1


def test_short_name_serving_handle_checks_arguments():
    """svdi_create / svdi_submit / svdi_poll / svdi_wait / svdi_destroy forward to the server entries:
    null handles and outputs are refused with SVDI_ERR_INVALID_ARGUMENT before any device call."""
    import ctypes
    from svdimager_b200 import api
    L = api.lib()
    P = ctypes.c_void_p
    L.svdi_create.argtypes = [P, P]
    L.svdi_submit.argtypes = [P, P, ctypes.c_size_t, ctypes.c_float, P, P]
    L.svdi_poll.argtypes = [P, ctypes.c_uint64, P]
    L.svdi_wait.argtypes = [P, ctypes.c_uint64, ctypes.c_double, P]
    L.svdi_destroy.argtypes = [P]
    L.svdi_destroy.restype = None
    opt = api.default_options()
    assert L.svdi_create(ctypes.addressof(opt), None) == 1
    done, ticket = ctypes.c_int(0), ctypes.c_uint64(0)
    assert L.svdi_submit(None, None, 16, 1e-3, None, ctypes.addressof(ticket)) == 1
    assert L.svdi_poll(None, 1, ctypes.addressof(done)) == 1
    assert L.svdi_wait(None, 1, 0.0, None) == 1
    assert L.svdi_last_error()
    L.svdi_destroy(None)  # a null handle is ignored


def test_fits_round_trip(tmp_path):
    from svdimager_b200 import fits
    a = np.arange(12, dtype=np.float32).reshape(3, 4) * 0.5
    p = str(tmp_path / "a.fits")
    fits.write_fits(p, a)
    assert np.array_equal(fits.read_fits(p), a)
    assert os.path.getsize(p) % 2880 == 0
    d = np.linspace(0, 1, 7)
    fits.write_fits(p, d)  # float64 -> BITPIX -64, read back as float
    assert np.allclose(fits.read_fits(p, np.float64), d)


def test_fits_sin_wcs_cards(tmp_path):
    from svdimager_b200 import fits
    p = str(tmp_path / "w.fits")
    a = np.zeros((8, 8), np.float32)
    fits.write_fits(p, a, extra_cards=fits.sin_wcs_cards(8, 1e-3, 150.0, -30.0))
    with open(p, "rb") as f:
        hdr, _ = fits.read_header(f.read())
    assert hdr["CTYPE1"] == "RA---SIN" and hdr["CTYPE2"] == "DEC--SIN" and hdr["BUNIT"] == "JY/BEAM"
    assert hdr["CRPIX1"] == 5.0 and hdr["CRVAL2"] == -30.0
    assert abs(hdr["CDELT1"] + np.degrees(1e-3)) < 1e-15 and abs(hdr["CDELT2"] - np.degrees(1e-3)) < 1e-15
    assert np.array_equal(fits.read_fits(p), a)


def test_cli_usage_exit_codes():
    b = os.path.join(ROOT, "svdimager_b200", "bin")
    r = subprocess.run([os.path.join(b, "sharedlibrary_gpu")], capture_output=True, text=True)
    assert r.returncode == 2 and "Usage" in r.stderr
    r = subprocess.run([os.path.join(b, "svd_integrated_imager_gpu"), "x"], capture_output=True, text=True)
    assert r.returncode == 2 and "Usage" in r.stderr
    r = subprocess.run([os.path.join(b, "svd_integrated_imager_gpu"), "missing", "0", "1e-3", "0", "o.fits"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Image_Size" in r.stderr


def test_bundle_reader_selects_time_groups(tmp_path):
    """Bundle reader (C++) groups rows by TIME like SVDIntegratedImager.cu:333-378; checked through
    the CLI's error path for an out-of-range snapshot index (no GPU needed)."""
    from svdimager_b200 import bundle, synth
    s0 = synth.make_snapshot("small", n_rows_limit=50, nchan=4, snapshot_index=0)
    s1 = synth.make_snapshot("small", n_rows_limit=50, nchan=4, snapshot_index=1)
    p = str(tmp_path / "b.ms")
    bundle.write_bundle(p, [s1, s0])  # TIME 1 then TIME 0: groups are sorted by TIME
    exe = os.path.join(ROOT, "svdimager_b200", "bin", "svd_integrated_imager_gpu")
    r = subprocess.run([exe, p, "64", "1e-3", "2", str(tmp_path / "o.fits")], capture_output=True, text=True)
    assert r.returncode == 1 and "Snapshot_Index is outside" in r.stderr


def test_autotune_candidates_and_beta():
    from svdimager_b200 import api, autotune
    assert abs(autotune.es_beta(8, 1.5) - autotune.REF_BETA) < 1e-12
    assert autotune.es_beta(12, 2.0) > autotune.es_beta(8, 2.0) > autotune.es_beta(8, 1.25)
    c = autotune.candidates()
    # W in {6, 8, 10, 12} x sigma in 4 values x (two FP32 tiles, plus the tensor core for W <= 8)
    assert len(c) == 4 * 4 * 2 + 2 * 4
    assert all(o["gridder"] == api.GRIDDER_FP32 or o["support"] <= 8 for o in c)
