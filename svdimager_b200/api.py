"""Python mirror of the svdimager_b200 C ABI (include/svdimager_b200.h).

Names follow the reference's entry points:
  FIpipe                          archive/pipe_interface.cpp:8, archive/FIPkernels.cu:679
  preprocess_measurement_set_gpu  SVDIntegratedImager.cu:76-79
  FIpipeDevice                    SVDIntegratedImager.cu:81-86
  free_device_preprocess_buffers  SVDIntegratedImager.cu:855-865
Errors raise SvdiError carrying the C status and message (the reference throws
std::runtime_error from the main path and reports nothing from FIpipe).

The compiled library is required: importing this module without it raises ImportError.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsvdimager_b200.so")

SVDI_OK = 0
KRULE_BUCKET, KRULE_MIN, KRULE_TARGET, KRULE_FIXED = 0, 1, 2, 3
EDGE_CLIP, EDGE_STRICT = 0, 1
COORD_FP64, COORD_REF32 = 0, 1
REPROJ_SII, REPROJ_FIPK = 0, 1
GRIDDER_FP32, GRIDDER_TC, GRIDDER_TC_BF16, GRIDDER_TC_I8 = 0, 1, 2, 3

# every function the C header declares (the ABI test checks they are all exported)
EXPORTED_SYMBOLS = (
    "svdi_last_error", "svdi_fipipe", "svdi_preprocess_measurement_set", "svdi_fipipe_device",
    "svdi_free_device_buffers", "svdi_default_options", "svdi_engine_create", "svdi_engine_destroy",
    "svdi_engine_image_host", "svdi_engine_image_device", "svdi_engine_fipipe_host",
    "svdi_engine_last_stats", "svdi_engine_buffer_size", "svdi_engine_copy_buffer",
    "svdi_kernel_launch_count", "svdi_bin_samples_noalloc", "svdi_server_create",
    "svdi_server_submit", "svdi_server_wait", "svdi_server_poll", "svdi_server_stats",
    "svdi_server_destroy", "svdi_engine_dft_pixels", "svdi_batch_create", "svdi_batch_launch",
    "svdi_batch_check", "svdi_batch_plan", "svdi_batch_mode", "svdi_batch_destroy", "svdi_copy_to_host", "_Z6FIpipePfS_S_S_S_mmf",
    "svdi_create", "svdi_submit", "svdi_poll", "svdi_wait", "svdi_destroy",
)
NOALLOC_MAX_KEYS = 16384

BUF_VIS_REAL, BUF_VIS_IMAG, BUF_Q, BUF_S, BUF_VIN, BUF_OFFSETS, BUF_RECORDS, BUF_RECORDS_S, \
    BUF_GRID, BUF_MOMENTS = range(10)
_BUF_DTYPE = {BUF_VIS_REAL: np.float32, BUF_VIS_IMAG: np.float32, BUF_Q: np.float64,
              BUF_S: np.float64, BUF_VIN: np.float64, BUF_OFFSETS: np.uint32,
              BUF_RECORDS: np.dtype([("xq", "<i4"), ("yq", "<i4"), ("vre", "<f4"), ("vim", "<f4")]),
              BUF_RECORDS_S: np.float32, BUF_GRID: np.complex64, BUF_MOMENTS: np.complex64}


class SvdiError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"svdimager_b200 error {status}: {message}")
        self.status = status
        self.message = message


class HostMS(ctypes.Structure):
    _fields_ = [
        ("num_rows", ctypes.c_size_t), ("num_channels", ctypes.c_size_t),
        ("num_samples", ctypes.c_size_t),
        ("uvw", ctypes.c_void_p), ("frequencies_hz", ctypes.c_void_p),
        ("vis0_real", ctypes.c_void_p), ("vis0_imag", ctypes.c_void_p),
        ("vis3_real", ctypes.c_void_p), ("vis3_imag", ctypes.c_void_p),
        ("flag0", ctypes.c_void_p), ("flag3", ctypes.c_void_p),
        ("weight0", ctypes.c_void_p), ("weight3", ctypes.c_void_p),
        ("array_center_x", ctypes.c_float),
    ]


class DeviceBuffers(ctypes.Structure):
    _fields_ = [
        ("d_bin", ctypes.c_void_p), ("d_vin", ctypes.c_void_p), ("d_vis_real", ctypes.c_void_p),
        ("d_vis_imag", ctypes.c_void_p), ("num_samples", ctypes.c_size_t),
        ("num_rows", ctypes.c_size_t), ("num_channels", ctypes.c_size_t),
        ("d_vin64", ctypes.c_void_p), ("d_q", ctypes.c_void_p), ("d_s", ctypes.c_void_p),
        ("d_stats", ctypes.c_void_p), ("internal", ctypes.c_void_p),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int), ("k_rule", ctypes.c_int), ("fixed_k", ctypes.c_int),
        ("target_error", ctypes.c_double), ("target_alpha", ctypes.c_double),
        ("edge_mode", ctypes.c_int), ("coord_mode", ctypes.c_int), ("reprojection", ctypes.c_int),
        ("support", ctypes.c_int), ("beta", ctypes.c_double), ("sigma", ctypes.c_double),
        ("tile", ctypes.c_int), ("gridder", ctypes.c_int), ("max_batch_slabs", ctypes.c_size_t),
        ("keep_grid", ctypes.c_int), ("presplat", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("num_samples", ctypes.c_size_t), ("num_gridded", ctypes.c_size_t),
        ("grid_size", ctypes.c_size_t), ("num_slabs", ctypes.c_int), ("num_terms", ctypes.c_int),
        ("num_planes", ctypes.c_int), ("r3_min", ctypes.c_double), ("r3_max", ctypes.c_double),
        ("max_abs_t3", ctypes.c_double), ("valid_pixels", ctypes.c_size_t),
        ("alpha_max", ctypes.c_double), ("slab_alpha_max", ctypes.c_double),
        ("vin", ctypes.c_double * 9), ("tile", ctypes.c_int), ("tile_cols", ctypes.c_int),
        ("used_tc", ctypes.c_int), ("num_keys", ctypes.c_int),
        ("slab_r3_min", ctypes.c_double), ("slab_width", ctypes.c_double),
        ("slab_half", ctypes.c_double), ("ms_total", ctypes.c_float),
        ("ms_preprocess", ctypes.c_float), ("ms_bin", ctypes.c_float), ("ms_grid", ctypes.c_float),
        ("ms_fft", ctypes.c_float), ("ms_image", ctypes.c_float),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "vin"}
        d["vin"] = list(self.vin)
        return d


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("slot", ctypes.c_int), ("num_samples", ctypes.c_size_t),
                ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """Load the compiled library; there is no fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"svdimager_b200 native library missing: {LIB_PATH} "
                              "(build it with `python -m svdimager_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        P, sz, f, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float, ctypes.c_int
        L.svdi_last_error.restype = ctypes.c_char_p
        L.svdi_fipipe.argtypes = [P, P, P, P, P, sz, sz, f]
        L.svdi_preprocess_measurement_set.argtypes = [ctypes.POINTER(HostMS), ctypes.POINTER(DeviceBuffers), i]
        L.svdi_fipipe_device.argtypes = [ctypes.POINTER(DeviceBuffers), P, sz, f]
        L.svdi_free_device_buffers.argtypes = [ctypes.POINTER(DeviceBuffers)]
        L.svdi_free_device_buffers.restype = None
        L.svdi_copy_to_host.argtypes = [P, P, sz]
        L.svdi_default_options.argtypes = [ctypes.POINTER(Options)]
        L.svdi_default_options.restype = None
        L.svdi_engine_create.argtypes = [ctypes.POINTER(Options), ctypes.POINTER(P)]
        L.svdi_engine_destroy.argtypes = [P]
        L.svdi_engine_destroy.restype = None
        L.svdi_engine_image_host.argtypes = [P, ctypes.POINTER(HostMS), sz, f, P]
        L.svdi_engine_image_device.argtypes = [P, ctypes.POINTER(HostMS), sz, f, P, P]
        L.svdi_engine_fipipe_host.argtypes = [P, P, P, P, P, P, sz, sz, f]
        L.svdi_engine_last_stats.argtypes = [P, ctypes.POINTER(Stats)]
        L.svdi_engine_buffer_size.argtypes = [P, i, ctypes.POINTER(sz)]
        L.svdi_engine_copy_buffer.argtypes = [P, i, P, sz]
        L.svdi_kernel_launch_count.restype = ctypes.c_uint64
        L.svdi_bin_samples_noalloc.argtypes = [P, P, P, sz, sz, f, i, f, P, P, sz, P]
        L.svdi_server_create.argtypes = [ctypes.POINTER(Options), i, sz, i, ctypes.POINTER(P)]
        L.svdi_server_submit.argtypes = [P, ctypes.POINTER(HostMS), sz, f, P, ctypes.POINTER(ctypes.c_uint64)]
        L.svdi_server_wait.argtypes = [P, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(RequestInfo)]
        L.svdi_server_poll.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(i)]
        L.svdi_server_stats.argtypes = [P, ctypes.POINTER(sz), ctypes.POINTER(sz), ctypes.POINTER(sz),
                                        ctypes.POINTER(ctypes.c_uint64)]
        L.svdi_server_destroy.argtypes = [P]
        L.svdi_server_destroy.restype = None
        L.svdi_engine_dft_pixels.argtypes = [P, P, P, sz, P]
        L.svdi_batch_create.argtypes = [P, ctypes.POINTER(HostMS), sz, sz, f, P, ctypes.POINTER(P)]
        L.svdi_batch_launch.argtypes = [P, P]
        L.svdi_batch_check.argtypes = [P]
        L.svdi_batch_plan.argtypes = [P, sz, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.svdi_batch_destroy.argtypes = [P]
        L.svdi_batch_mode.argtypes = [P]
        L.svdi_batch_destroy.restype = None
        _lib = L
    return _lib


def _check(status: int):
    if status != SVDI_OK:
        raise SvdiError(status, lib().svdi_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def kernel_launch_count() -> int:
    return int(lib().svdi_kernel_launch_count())


def default_options(**kw) -> Options:
    o = Options()
    lib().svdi_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k!r}")
        setattr(o, k, v)
    return o


def archive_options(**kw) -> Options:
    """Options of the archive FIpipe path (smallest K in 1..32, trigonometric SIN)."""
    base = dict(k_rule=KRULE_MIN, reprojection=REPROJ_FIPK)
    base.update(kw)
    return default_options(**base)


_HOST_FIELDS = (("uvw", np.float32), ("frequencies_hz", np.float32), ("vis0_real", np.float32),
                ("vis0_imag", np.float32), ("vis3_real", np.float32), ("vis3_imag", np.float32),
                ("flag0", np.uint8), ("flag3", np.uint8), ("weight0", np.float32),
                ("weight3", np.float32))


def host_ms(snap):
    """(HostMS, keep-alive list) for a synth.Snapshot-like object with numpy fields."""
    keep = []
    h = HostMS()
    h.num_rows, h.num_channels = snap.num_rows, snap.num_channels
    h.num_samples = snap.num_rows * snap.num_channels
    for name, dt in _HOST_FIELDS:
        a = np.ascontiguousarray(getattr(snap, name), dtype=dt)
        keep.append(a)
        setattr(h, name, a.ctypes.data)
    h.array_center_x = float(snap.array_center_x)
    return h, keep


def device_ms(num_rows, num_channels, tensors: dict, array_center_x: float):
    """HostMS descriptor whose pointers are DEVICE addresses (torch tensors on cuda)."""
    h = HostMS()
    h.num_rows, h.num_channels = num_rows, num_channels
    h.num_samples = num_rows * num_channels
    for name, _ in _HOST_FIELDS:
        setattr(h, name, tensors[name].data_ptr())
    h.array_center_x = float(array_center_x)
    return h


class Engine:
    """Device-resident imaging engine (grids, plans and bins stay on the GPU between calls)."""

    def __init__(self, options: Optional[Options] = None, **kw):
        o = options if options is not None else default_options(**kw)
        h = ctypes.c_void_p()
        _check(lib().svdi_engine_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.options = o

    def close(self):
        if getattr(self, "_h", None):
            lib().svdi_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def image(self, snap, image_size: Optional[int] = None, cell_size: Optional[float] = None,
              out: Optional[np.ndarray] = None) -> np.ndarray:
        """Main path from host snapshot arrays to a host image [N][N] float32."""
        N = int(snap.image_size if image_size is None else image_size)
        cell = float(snap.cell_size if cell_size is None else cell_size)
        h, keep = host_ms(snap)
        if out is None:
            out = np.zeros((N, N), np.float32)
        _check(lib().svdi_engine_image_host(self._h, ctypes.byref(h), N, cell, _ptr(out)))
        return out

    def image_device(self, dev_ms: HostMS, image_size: int, cell_size: float, out_ptr: int,
                     stream_ptr: int = 0):
        _check(lib().svdi_engine_image_device(self._h, ctypes.byref(dev_ms), int(image_size),
                                              float(cell_size), ctypes.c_void_p(out_ptr),
                                              ctypes.c_void_p(stream_ptr)))

    def fipipe(self, visreal, visimag, bin_, vin, image_size: int, cell_size: float,
               out: Optional[np.ndarray] = None) -> np.ndarray:
        """Archive-semantics imaging of one quartet on this engine; `out`, when given, is a
        C-contiguous float32 [image_size][image_size] array that receives the image."""
        vr = np.ascontiguousarray(visreal, np.float32)
        vi = np.ascontiguousarray(visimag, np.float32)
        b = np.ascontiguousarray(bin_, np.float32).reshape(-1)
        v = np.ascontiguousarray(vin, np.float32).reshape(-1)
        if out is None:
            out = np.zeros((image_size, image_size), np.float32)
        elif (out.dtype != np.float32 or out.shape != (image_size, image_size)
              or not out.flags["C_CONTIGUOUS"]):
            raise SvdiError(1, "out must be a C-contiguous float32 [image_size][image_size] array")
        _check(lib().svdi_engine_fipipe_host(self._h, _ptr(vr), _ptr(vi), _ptr(b), _ptr(v), _ptr(out),
                                             vr.shape[0], int(image_size), float(cell_size)))
        return out

    def buffer(self, which: int) -> np.ndarray:
        """Copy of an intermediate device buffer of the last call (SVDI_BUF_*)."""
        n = ctypes.c_size_t()
        _check(lib().svdi_engine_buffer_size(self._h, which, ctypes.byref(n)))
        dt = np.dtype(_BUF_DTYPE[which])
        out = np.empty(n.value // dt.itemsize, dt)
        if out.nbytes:
            _check(lib().svdi_engine_copy_buffer(self._h, which, out.ctypes.data_as(ctypes.c_void_p),
                                                 out.nbytes))
        return out

    def stats(self) -> dict:
        s = Stats()
        _check(lib().svdi_engine_last_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    def dft_pixels(self, px, py) -> np.ndarray:
        """FP64 direct DFT of the last snapshot at pixels (px, py): the rotated-frame image value
        before reprojection (compare with an image made with presplat=1); NaN outside the
        projection."""
        x = np.ascontiguousarray(px, np.int64)
        y = np.ascontiguousarray(py, np.int64)
        out = np.zeros(len(x), np.float64)
        _check(lib().svdi_engine_dft_pixels(self._h, _ptr(x), _ptr(y), len(x), _ptr(out)))
        return out


class Batch:
    """Many device-resident snapshots imaged by one CUDA-graph launch (svdi_batch_*). Creating it
    images every snapshot once (recording each snapshot's plan) and captures the graph; launch()
    replays it. `snapshots` are device descriptors (device_ms); `images_ptr` is a device buffer of
    len(snapshots) x N x N floats. Keep the engine, the snapshots' arrays and the images alive
    while the batch exists."""

    def __init__(self, engine: "Engine", snapshots, image_size: int, cell_size: float, images_ptr: int):
        arr = (HostMS * len(snapshots))(*snapshots)
        h = ctypes.c_void_p()
        _check(lib().svdi_batch_create(engine._h, arr, len(snapshots), int(image_size), float(cell_size),
                                       ctypes.c_void_p(images_ptr), ctypes.byref(h)))
        self._h = h
        self._arr = arr
        self.engine = engine
        self.num = len(snapshots)

    def launch(self, stream_ptr: int = 0):
        _check(lib().svdi_batch_launch(self._h, ctypes.c_void_p(stream_ptr)))

    def check(self):
        _check(lib().svdi_batch_check(self._h))

    def plan(self, index: int):
        ns, nt = ctypes.c_int(), ctypes.c_int()
        _check(lib().svdi_batch_plan(self._h, int(index), ctypes.byref(ns), ctypes.byref(nt)))
        return {"num_slabs": ns.value, "num_terms": nt.value}

    @property
    def wide(self) -> bool:
        """True when every stage runs over all snapshots at once (one gridder launch per order)."""
        return lib().svdi_batch_mode(self._h) == 1

    def close(self):
        if getattr(self, "_h", None):
            lib().svdi_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def FIpipe(Visreal, Visimag, Bin, Vin, image_size: int, cell_size: float,
           num_baselines: Optional[int] = None) -> np.ndarray:
    """Archive entry point (archive/FIPkernels.cu:679). Returns the dirty image [N][N]."""
    vr = np.ascontiguousarray(Visreal, np.float32)
    vi = np.ascontiguousarray(Visimag, np.float32)
    b = np.ascontiguousarray(Bin, np.float32).reshape(-1)
    v = np.ascontiguousarray(Vin, np.float32).reshape(-1)
    n = int(num_baselines if num_baselines is not None else vr.shape[0])
    if vr.shape[0] < n or vi.shape[0] < n or b.shape[0] < 3 * n or v.shape[0] < 9:
        raise SvdiError(1, "input arrays shorter than num_baselines")
    out = np.zeros((image_size, image_size), np.float32)
    _check(lib().svdi_fipipe(_ptr(vr), _ptr(vi), _ptr(b), _ptr(v), _ptr(out), n, int(image_size),
                             float(cell_size)))
    return out


class PreprocessBuffers:
    """DevicePreprocessBuffers: owns the device arrays made by preprocess_measurement_set_gpu."""

    def __init__(self, buf: DeviceBuffers, keep):
        self.buf = buf
        self._keep = keep

    def free(self):
        if self.buf is not None and self.buf.internal:
            lib().svdi_free_device_buffers(ctypes.byref(self.buf))
        self.buf = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def preprocess_measurement_set_gpu(snap, want_bin: bool = False) -> PreprocessBuffers:
    h, keep = host_ms(snap)
    b = DeviceBuffers()
    _check(lib().svdi_preprocess_measurement_set(ctypes.byref(h), ctypes.byref(b), int(want_bin)))
    return PreprocessBuffers(b, keep)


def copy_to_host(out: np.ndarray, device_ptr: int) -> np.ndarray:
    """Fill the contiguous numpy array `out` from a device address (svdi_copy_to_host)."""
    if not out.flags.c_contiguous:
        raise ValueError("out must be C-contiguous")
    _check(lib().svdi_copy_to_host(_ptr(out), ctypes.c_void_p(device_ptr), out.nbytes))
    return out


def FIpipeDevice(buffers: PreprocessBuffers, image_size: int, cell_size: float) -> np.ndarray:
    out = np.zeros((image_size, image_size), np.float32)
    _check(lib().svdi_fipipe_device(ctypes.byref(buffers.buf), _ptr(out), int(image_size), float(cell_size)))
    return out


def free_device_preprocess_buffers(buffers: PreprocessBuffers):
    buffers.free()


class Server:
    """Continuous-batching imaging server (svdi_server_*): `num_slots` resident engines, one
    worker thread each; requests are admitted by free slot and HBM budget and overlap on the GPU.
    submit() keeps the snapshot's arrays and the output image alive until wait() returns."""

    def __init__(self, options: Optional[Options] = None, num_slots: int = 4, hbm_budget: int = 0,
                 fault_every: int = 0, **kw):
        o = options if options is not None else default_options(**kw)
        h = ctypes.c_void_p()
        _check(lib().svdi_server_create(ctypes.byref(o), int(num_slots), int(hbm_budget), int(fault_every),
                                        ctypes.byref(h)))
        self._h = h
        self._pending = {}

    def submit(self, snap, image_size: Optional[int] = None, cell_size: Optional[float] = None,
               out: Optional[np.ndarray] = None) -> int:
        """Queue one snapshot; `out` (float32 [N][N], e.g. in pinned memory) receives the image,
        a new array when omitted."""
        N = int(snap.image_size if image_size is None else image_size)
        cell = float(snap.cell_size if cell_size is None else cell_size)
        h, keep = host_ms(snap)
        if out is None:
            out = np.zeros((N, N), np.float32)
        elif out.dtype != np.float32 or out.shape != (N, N) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of N x N")
        t = ctypes.c_uint64()
        _check(lib().svdi_server_submit(self._h, ctypes.byref(h), N, cell, _ptr(out), ctypes.byref(t)))
        self._pending[t.value] = (h, keep, out)
        return t.value

    def wait(self, ticket: int, timeout_s: float = 0.0):
        """(image, info dict); raises SvdiError when the request failed."""
        info = RequestInfo()
        st = lib().svdi_server_wait(self._h, ctypes.c_uint64(ticket), float(timeout_s), ctypes.byref(info))
        _, _, out = self._pending.pop(ticket, (None, None, None))
        _check(st)
        return out, info.as_dict()

    def stats(self) -> dict:
        q, u, b, a = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_uint64()
        _check(lib().svdi_server_stats(self._h, ctypes.byref(q), ctypes.byref(u), ctypes.byref(b),
                                       ctypes.byref(a)))
        return {"queued": q.value, "hbm_in_use": u.value, "hbm_budget": b.value, "admitted": a.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().svdi_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bin_samples_noalloc(d_bin: int, d_vis_real: int, d_vis_imag: int, num_samples: int,
                        image_size: int, cell_size: float, tile: int, inv_det: float,
                        d_records: int, d_offsets: int, offsets_capacity: int, stream: int = 0):
    """Allocation-free tile binning on DEVICE pointers (svdi_bin_samples_noalloc): for callers
    that may not allocate device memory while they run. Scratch lives in a fixed static device
    array (at most NOALLOC_MAX_KEYS tile keys); overlapping calls on one device race."""
    _check(lib().svdi_bin_samples_noalloc(
        ctypes.c_void_p(d_bin), ctypes.c_void_p(d_vis_real), ctypes.c_void_p(d_vis_imag),
        int(num_samples), int(image_size), float(cell_size), int(tile), float(inv_det),
        ctypes.c_void_p(d_records), ctypes.c_void_p(d_offsets), int(offsets_capacity),
        ctypes.c_void_p(stream)))
