"""ORACLE — test infrastructure only.

Python side of the CPU restatement of the reference snapshot imager (egbdfX/SVDimager): ctypes
bindings of ``liboracle.so`` (oracle.c), the reference's host-side Chebyshev/slab selection and the
inverse FFT (numpy, FP64). Only tests/, the smoke check in __graft_entry__.py and bench.py's CPU
legs import this module; the product never does.

Reference files cited below, relative to the reference project root:
  SII  = SVDIntegratedImager.cu, FIPK = archive/FIPkernels.cu, MFS = archive/SVD_MFS.py.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libfipk_ref.so")

# Constants of the reference imager (SII:1233-1235, SII:1510-1512, SII:35-37)
REF_SUPPORT = 8
REF_BETA = 15.3704324328
CHEB_MAX_MOMENTS = 32
CHEB_TARGET_ERROR = 1.0e-2
CHEB_TARGET_ALPHA = 10.0

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(HERE, "oracle.c")):
            build()
        L = ctypes.CDLL(LIB_PATH)
        d, f, i64, u8, l, i = (ctypes.c_double, ctypes.c_float, ctypes.c_int64, ctypes.c_uint8,
                               ctypes.c_long, ctypes.c_int)
        P = ctypes.c_void_p
        L.orc_collapse.argtypes = [l] + [P] * 10
        L.orc_preprocess64.argtypes = [l, l, P, P, f, P, P, P, P]
        L.orc_expand_coords.argtypes = [l, l, P, P, P]
        L.orc_es.restype = d
        L.orc_es.argtypes = [d, d]
        L.orc_es_correction.argtypes = [l, l, i, d, P]
        L.orc_tile_keys.argtypes = [l, P, d, i, l, i, i, i, l, i, i, d, d, d, P, P, P, P]
        L.orc_grid.argtypes = [l, P, P, P, d, i, l, i, d, i, i, d, d, d, d, i, P]
        L.orc_bessel_j.argtypes = [d, i, P]
        L.orc_bessel_series_f32.argtypes = [f, i, P]
        L.orc_recombine.argtypes = [P, l, l, d, P, i, i, d, d, d, P, d, l, l, P]
        L.orc_dft_pixels.argtypes = [l, P, P, P, P, d, d, P, l, d, l, P, P, P]
        L.orc_dft_pixels_sep.argtypes = [l, l, P, P, P, P, P, d, d, P, l, d, l, P, P, P]
        L.orc_reproject_sii.argtypes = [P, l, d, P, l, l, P]
        L.orc_reproject_fipk.argtypes = [P, l, d, P, l, l, P]
        L.orc_t3_stats.argtypes = [P, l, d, P, P]
        L.orc_cheb_errors.argtypes = [d, i, i, i, P]
        L.orc_num_threads.restype = i
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# ------------------------------------------------------------------------------------------
# pre-processing
# ------------------------------------------------------------------------------------------
def collapse(snap):
    """Flag/weight polarisation collapse, FP32 (SII:588-617)."""
    n = snap.num_samples
    outr = np.empty(n, np.float32)
    outi = np.empty(n, np.float32)
    lib().orc_collapse(n, *[_p(_c(getattr(snap, k), dt)) for k, dt in (
        ("vis0_real", np.float32), ("vis0_imag", np.float32), ("vis3_real", np.float32),
        ("vis3_imag", np.float32), ("flag0", np.uint8), ("flag3", np.uint8),
        ("weight0", np.float32), ("weight3", np.float32))], _p(outr), _p(outi))
    return outr, outi


def preprocess64(snap):
    """FP64 SVD rotation (SII:409-586). Returns vin (3x3 row-major), q [rows,3], s [chan]."""
    vin = np.zeros(9)
    q = np.zeros((snap.num_rows, 3))
    s = np.zeros(snap.num_channels)
    ev = np.zeros(3)
    lib().orc_preprocess64(snap.num_rows, snap.num_channels, _p(_c(snap.uvw, np.float32)),
                           _p(_c(snap.frequencies_hz, np.float32)), snap.array_center_x,
                           _p(vin), _p(q), _p(s), _p(ev))
    return vin.reshape(3, 3), q, s, ev


def expand_coords(q, s):
    nrows, nch = q.shape[0], s.shape[0]
    r = np.empty((nrows * nch, 3))
    lib().orc_expand_coords(nrows, nch, _p(_c(q, np.float64)), _p(_c(s, np.float64)), _p(r))
    return r


# ------------------------------------------------------------------------------------------
# Chebyshev / slab selection (host side of the reference)
# ------------------------------------------------------------------------------------------
def cheb_errors(amax, na, ns, kmax=CHEB_MAX_MOMENTS):
    err = np.zeros(kmax)
    lib().orc_cheb_errors(float(amax), na, ns, kmax, _p(err))
    return err


def t3_stats(vin, N, cell):
    m = ctypes.c_double(0.0)
    v = ctypes.c_long(0)
    lib().orc_t3_stats(_p(_c(vin, np.float64).reshape(-1)), N, float(cell), ctypes.byref(m),
                       ctypes.byref(v))
    return m.value, v.value


@dataclass
class SlabConfig:
    r3_min: float
    r3_max: float
    max_abs_t3: float
    alpha_max: float
    num_slabs: int
    slab_width: float
    slab_half: float
    inv_half: float
    slab_alpha_max: float
    K: int


def slab_config_sii(r3, vin, N, cell, target_alpha=CHEB_TARGET_ALPHA, k_rule="bucket"):
    """SII:926-991 (finish_host_chebyshev_selection, make_chebyshev_slab_config) and the bucket
    choice of K in {8,16,24,32} at sampled error <= 1e-2 (SII:1577-1603; 257 x 1024 samples)."""
    r3_min, r3_max = float(np.min(r3)), float(np.max(r3))
    mt3, _ = t3_stats(vin, N, cell)
    half_range = max(0.5 * (r3_max - r3_min), 1.0e-6)
    alpha_max = 2.0 * math.pi * mt3 * half_range
    r3_range = max(r3_max - r3_min, 2.0e-6)
    nslab = max(1, int(math.ceil(max(alpha_max, 0.0) / target_alpha)))
    width = r3_range / nslab
    slab_half = max(0.5 * width, 1.0e-6)
    slab_alpha = 2.0 * math.pi * mt3 * slab_half
    if k_rule == "bucket":
        err = cheb_errors(slab_alpha, 257, 1024)
        K = CHEB_MAX_MOMENTS
        for kb in (8, 16, 24, 32):
            if err[kb - 1] <= CHEB_TARGET_ERROR:
                K = kb
                break
    else:
        K = int(k_rule)
    return SlabConfig(r3_min, r3_max, mt3, alpha_max, nslab, width, slab_half, 1.0 / slab_half,
                      slab_alpha, K)


def bessel_j(x, nmax):
    """J_0(x) .. J_nmax(x) in FP64 (orc_bessel_j, Miller's recurrence)."""
    j = np.zeros(nmax + 1)
    lib().orc_bessel_j(float(x), int(nmax), _p(j))
    return j


def truncation_bound(a, K):
    """Jacobi-Anger truncation error bound on |s| <= 1 with K terms kept: 2 sum_{n>=K} |J_n(a)|."""
    j = bessel_j(a, min(199, K + 60 + int(abs(a))))
    return 2.0 * float(np.sum(np.abs(j[K:])))


def k_for_target(a, target, kmax=64):
    for K in range(1, kmax + 1):
        if truncation_bound(a, K) <= target:
            return K
    return -1


def slab_config_target(r3, vin, N, cell, target_error=1e-6):
    """Error-target rule of the B200 engine (not in the reference): the slab count n in 1..64 that
    minimises the moment planes n * K (on ties the larger n, i.e. the smaller K), K the smallest
    order whose truncation bound at the slab's alpha is <= target_error; slab geometry as
    SII:973-991."""
    r3_min, r3_max = float(np.min(r3)), float(np.max(r3))
    mt3, _ = t3_stats(vin, N, cell)
    half_range = max(0.5 * (r3_max - r3_min), 1.0e-6)
    alpha_max = 2.0 * math.pi * mt3 * half_range
    r3_range = max(r3_max - r3_min, 2.0e-6)
    best_n, best_p = 1, 1 << 30
    for n in range(1, 65):
        h = max(0.5 * r3_range / n, 1.0e-6)
        K = k_for_target(2.0 * math.pi * mt3 * h, target_error)
        if K < 0:
            continue
        if n * K <= best_p:  # equal plane counts: the smaller K (more slabs)
            best_p, best_n = n * K, n
        if K == 1:
            break
    width = r3_range / best_n
    slab_half = max(0.5 * width, 1.0e-6)
    slab_alpha = 2.0 * math.pi * mt3 * slab_half
    K = k_for_target(slab_alpha, target_error)
    return SlabConfig(r3_min, r3_max, mt3, alpha_max, best_n, width, slab_half, 1.0 / slab_half,
                      slab_alpha, K)


def slab_config_fipk(r3, vin, N, cell):
    """FIPK:320-366 compute_host_chebyshev_selection: one slab centred on the r3 range, K = the
    smallest kept-term count in 1..32 whose sampled error (513 x 2048, FP64) is <= 1e-2."""
    r3_min, r3_max = float(np.min(r3)), float(np.max(r3))
    centre = 0.5 * (r3_max + r3_min)
    half = max(0.5 * (r3_max - r3_min), 1.0e-6)
    mt3, _ = t3_stats(vin, N, cell)
    alpha_max = 2.0 * math.pi * mt3 * half
    err = cheb_errors(alpha_max, 513, 2048)
    K = CHEB_MAX_MOMENTS
    for k in range(1, CHEB_MAX_MOMENTS + 1):
        if err[k - 1] <= CHEB_TARGET_ERROR:
            K = k
            break
    return SlabConfig(centre - half, r3_max, mt3, alpha_max, 1, 2.0 * half, half, 1.0 / half,
                      alpha_max, K)


# ------------------------------------------------------------------------------------------
# imaging
# ------------------------------------------------------------------------------------------
def grid_size_for(N, sigma=1.5):
    """G = ceil(1.5 N) (SII:1510; FIPK:704 computes the same through a float)."""
    return int(math.ceil(N * sigma - 1e-9)) if sigma != 1.5 else (3 * N + 1) // 2


def es_correction(N, G, W=REF_SUPPORT, beta=REF_BETA):
    phi = np.zeros(N // 2 + 1)
    lib().orc_es_correction(N // 2, G, W, beta, _p(phi))
    return phi


def tile_keys(r, scale, G, W, T, edge_mode, sc: SlabConfig, coord_mode=0, records=False,
              T2=None, ntile2=None):
    """Per-sample tile key (-1 = dropped); with records=True also the record coordinates
    (xq, yq) and the Chebyshev argument of the B200 binning contract. Tiles are T rows by
    T2 columns (default square) with ntile2 tile columns per tile row (default ceil(G / T2))."""
    n = r.shape[0]
    T2 = T if T2 is None else T2
    ntile2 = (G + T2 - 1) // T2 if ntile2 is None else ntile2
    keys = np.empty(n, np.int64)
    xq = np.zeros(n, np.int32) if records else None
    yq = np.zeros(n, np.int32) if records else None
    sa = np.zeros(n, np.float32) if records else None
    lib().orc_tile_keys(n, _p(_c(r, np.float64)), float(scale), coord_mode, G, W, T,
                        T2, ntile2, edge_mode, sc.num_slabs, sc.r3_min, sc.slab_width, sc.inv_half, _p(keys),
                        _p(xq), _p(yq), _p(sa))
    return (keys, xq, yq, sa) if records else keys


def grid(r, vr, vi, scale, G, sc: SlabConfig, inv_det, W=REF_SUPPORT, beta=REF_BETA, edge_mode=0,
         coord_mode=0):
    P = sc.num_slabs * sc.K
    planes = np.zeros((P, G, G), np.complex128)
    lib().orc_grid(r.shape[0], _p(_c(r, np.float64)), _p(_c(vr, np.float32)),
                   _p(_c(vi, np.float32)), float(scale), coord_mode, G, W, beta, sc.K, sc.num_slabs,
                   sc.r3_min, sc.slab_width, sc.inv_half, float(inv_det), edge_mode, _p(planes))
    return planes


def inverse_fft(planes):
    """Unnormalised inverse 2-D DFT of every plane, as cufftExecC2C(CUFFT_INVERSE) (SII:1713).
    FP64, on all host cores (scipy's pocketfft with workers=-1)."""
    import scipy.fft
    G = planes.shape[-1]
    return scipy.fft.ifft2(planes, axes=(-2, -1), workers=-1) * (G * G)


def recombine(moments, N, cell, vin, sc: SlabConfig, phi, n_total, rows=None):
    """Pre-splat image R [N][N]; rows = (y0, y1) computes those image rows only (others 0)."""
    G = moments.shape[-1]
    R = np.zeros((N, N))
    y0, y1 = rows or (0, N)
    lib().orc_recombine(_p(_c(moments, np.complex128)), G, N, float(cell),
                        _p(_c(vin, np.float64).reshape(-1)), sc.K, sc.num_slabs, sc.r3_min,
                        sc.slab_width, sc.slab_half, _p(_c(phi, np.float64)), float(n_total),
                        int(y0), int(y1), _p(R))
    return R


def reproject(R, N, cell, vin, variant="sii", rows=None):
    """Bilinear splat of the valid pixels of R (rows = (y0, y1): those pixel rows only)."""
    out = np.zeros((N, N))
    y0, y1 = rows or (0, N)
    fn = lib().orc_reproject_sii if variant == "sii" else lib().orc_reproject_fipk
    fn(_p(_c(R, np.float64)), N, float(cell), _p(_c(vin, np.float64).reshape(-1)), int(y0), int(y1),
       _p(out))
    return out


def inclusion_mask(r, scale, G, W=REF_SUPPORT, edge_mode=1, coord_mode=0):
    """Samples the gridder keeps: any footprint cell on the grid (edge_mode 0) or the whole
    footprint on the grid (edge_mode 1)."""
    sc = SlabConfig(0, 0, 0, 0, 1, 1.0, 0.5, 2.0, 0, 1)
    return (tile_keys(r, scale, G, W, 16, edge_mode, sc, coord_mode) >= 0).astype(np.uint8)


def dft_pixels(r, vr, vi, inv_det, n_total, vin, N, cell, px, py, include=None):
    out = np.zeros(len(px))
    lib().orc_dft_pixels(r.shape[0], _p(_c(r, np.float64)), _p(_c(vr, np.float32)),
                         _p(_c(vi, np.float32)), _p(include), float(inv_det), float(n_total),
                         _p(_c(vin, np.float64).reshape(-1)), N, float(cell), len(px),
                         _p(_c(px, np.int64)), _p(_c(py, np.int64)), _p(out))
    return out


def dft_pixels_sep(q, s, vr, vi, inv_det, n_total, vin, N, cell, px, py, include=None):
    out = np.zeros(len(px))
    lib().orc_dft_pixels_sep(q.shape[0], s.shape[0], _p(_c(q, np.float64)),
                             _p(_c(s, np.float64)), _p(_c(vr, np.float32)),
                             _p(_c(vi, np.float32)), _p(include), float(inv_det), float(n_total),
                             _p(_c(vin, np.float64).reshape(-1)), N, float(cell), len(px),
                             _p(_c(px, np.int64)), _p(_c(py, np.int64)), _p(out))
    return out


@dataclass
class OracleImage:
    image: np.ndarray        # final reprojected image [N][N]
    pre: np.ndarray          # pre-splat rotated-frame image R [N][N] (NaN = invalid)
    vin: np.ndarray
    sc: SlabConfig
    G: int
    r: np.ndarray            # per-sample FP64 coordinates
    vr: np.ndarray
    vi: np.ndarray


def image_fipk(visr, visi, bin_, vin, N, cell, edge_mode=0, W=REF_SUPPORT, beta=REF_BETA,
               coord_mode=1):
    """Archive FIpipe (FIPK:679-911) on host arrays: float Bin [N_s][3], float Vin 3x3."""
    vin64 = np.asarray(vin, np.float32).astype(np.float64).reshape(3, 3)
    r = np.asarray(bin_, np.float32).astype(np.float64).reshape(-1, 3)
    n = r.shape[0]
    G = grid_size_for(N)
    scale = float(np.float32(cell)) * G
    sc = slab_config_fipk(np.asarray(bin_, np.float32).reshape(-1, 3)[:, 2], vin64, N, cell)
    inv_det = 1.0 / abs(vin64[0, 0] * vin64[1, 1] - vin64[0, 1] * vin64[1, 0])
    planes = grid(r, visr, visi, scale, G, sc, inv_det, W, beta, edge_mode, coord_mode)
    moments = inverse_fft(planes)
    phi = es_correction(N, G, W, beta)
    R = recombine(moments, N, float(np.float32(cell)), vin64, sc, phi, n)
    img = reproject(R, N, float(np.float32(cell)), vin64, "fipk")
    return OracleImage(img, R, vin64, sc, G, r, visr, visi)


def image_sii(snap, N=None, cell=None, edge_mode=0, k_rule="bucket", target_alpha=CHEB_TARGET_ALPHA,
              W=REF_SUPPORT, beta=REF_BETA, sigma=1.5, coord_mode=0):
    """Main path: preprocess_measurement_set_gpu + FIpipeDevice (SII:635-853, SII:1498-1761),
    with FP64 coordinates."""
    N = N or snap.image_size
    cell = cell or snap.cell_size
    vr, vi = collapse(snap)
    vin, q, s, _ = preprocess64(snap)
    r = expand_coords(q, s)
    n = r.shape[0]
    G = grid_size_for(N, sigma)
    cell64 = float(np.float32(cell))
    scale = cell64 * G
    sc = slab_config_sii(r[:, 2], vin, N, cell64, target_alpha, k_rule)
    inv_det = 1.0 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    planes = grid(r, vr, vi, scale, G, sc, inv_det, W, beta, edge_mode, coord_mode)
    moments = inverse_fft(planes)
    phi = es_correction(N, G, W, beta)
    R = recombine(moments, N, cell64, vin, sc, phi, n)
    img = reproject(R, N, cell64, vin, "sii")
    return OracleImage(img, R, vin, sc, G, r, vr, vi)


REF_PRECISE_LIB_PATH = os.path.join(HERE, "_ref", "libfipk_ref_precise.so")


def load_reference_fipipe(precise=False):
    """The reference's own archive FIpipe (compiled from archive/FIPkernels.cu for sm_100a by
    oracle/Makefile; precise=True: the build without --use_fast_math) or None when it was not
    built. Runs on the GPU only."""
    path = REF_PRECISE_LIB_PATH if precise else REF_LIB_PATH
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    fn = getattr(L, "_Z6FIpipePfS_S_S_S_mmf")  # int FIpipe(float*,float*,float*,float*,float*,size_t,size_t,float)
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_float]
    return fn


def run_reference_fipipe(visr, visi, bin_, vin, N, cell, precise=False):
    fn = load_reference_fipipe(precise)
    if fn is None:
        raise RuntimeError("reference library not built (make -C oracle ref)")
    vr = _c(visr, np.float32).copy()
    vi = _c(visi, np.float32).copy()
    b = _c(bin_, np.float32).reshape(-1).copy()
    v = _c(vin, np.float32).reshape(-1).copy()
    out = np.zeros(N * N, np.float32)
    fn(_p(vr), _p(vi), _p(b), _p(v), _p(out), vr.shape[0], N, float(cell))
    return out.reshape(N, N)


def rel_rms(a, b, mask=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is None:
        mask = np.isfinite(a) & np.isfinite(b)
    d = a[mask] - b[mask]
    return float(np.sqrt(np.sum(d * d) / np.sum(b[mask] * b[mask])))
