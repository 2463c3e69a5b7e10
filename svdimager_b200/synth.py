"""Deterministic synthetic snapshots for the imaging configurations.

A snapshot is the content of one TIME group of a Measurement Set as the reference's reader
delivers it (``HostMeasurementSetData``, SVDIntegratedImager.cu:39-54): ``num_rows`` baselines x
``num_channels`` channels, flattened channel-major (``idx = row + chan * num_rows``,
SVDIntegratedImager.cu:90-92), with polarisations 0 and 3 (XX, YY), their FLAG and
WEIGHT_SPECTRUM, float UVW per row, float channel frequencies and ARRAY_CENTER.x.

No real Measurement Set is available, so every configuration is generated from a seeded
``numpy.random.PCG64`` stream (seed 20261203 + config index):

* station layouts (east, north, up) in metres, site latitude -30 deg;
* uvw by the standard (hour angle, declination) rotation of the equatorial baseline vectors;
* a sky of point sources, XX = YY = sum S exp(-2 pi i (u l + v m + w (n - 1))) plus complex
  Gaussian noise (sigma = 0.05 Jy per polarisation);
* WEIGHT_SPECTRUM ~ U[0.5, 1] per polarisation, row- or sample-level flags.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional

import numpy as np

C_LIGHT = 299792458.0
SEED_BASE = 20261203
SITE_LATITUDE = math.radians(-30.0)
ARRAY_CENTER = (5.1e6, 2.0e6, -3.2e6)
EARTH_RADIUS = 6.371e6


@dataclasses.dataclass
class Snapshot:
    """One TIME group, field for field like the reference's HostMeasurementSetData."""

    num_rows: int
    num_channels: int
    uvw: np.ndarray            # float32 [num_rows, 3]
    frequencies_hz: np.ndarray  # float32 [num_channels]
    vis0_real: np.ndarray      # float32 [num_samples], idx = row + chan * num_rows
    vis0_imag: np.ndarray
    vis3_real: np.ndarray
    vis3_imag: np.ndarray
    flag0: np.ndarray          # uint8 [num_samples]
    flag3: np.ndarray
    weight0: np.ndarray        # float32 [num_samples]
    weight3: np.ndarray
    array_center_x: float
    image_size: int = 256
    cell_size: float = 4e-4
    time: float = 0.0
    sources: Optional[np.ndarray] = None   # [nsrc, 3]: flux, l, m
    uvw64: Optional[np.ndarray] = None     # float64 uvw before the float cast

    @property
    def num_samples(self) -> int:
        return self.num_rows * self.num_channels

    def host_bytes(self) -> int:
        """Bytes of the host arrays a device upload moves."""
        return sum(a.nbytes for a in self.arrays().values())

    def arrays(self) -> Dict[str, np.ndarray]:
        return {k: getattr(self, k) for k in (
            "uvw", "frequencies_hz", "vis0_real", "vis0_imag", "vis3_real", "vis3_imag",
            "flag0", "flag3", "weight0", "weight3")}


# ------------------------------------------------------------------------------------------
# station layouts
# ------------------------------------------------------------------------------------------
def _disk(rng, n, radius):
    r = radius * np.sqrt(rng.random(n))
    th = 2 * np.pi * rng.random(n)
    return np.stack([r * np.cos(th), r * np.sin(th)], axis=1)


def _log_arms(rng, n, r_min, r_max):
    r = np.exp(np.linspace(np.log(r_min), np.log(r_max), n))
    th = 2 * np.pi * rng.random(n)
    return np.stack([r * np.cos(th), r * np.sin(th)], axis=1)


def station_layout(kind: str, rng: np.random.Generator, heights: bool = False) -> np.ndarray:
    """East/north/up station positions in metres.

    ``disk128``: 128 stations uniform in a 1.5 km-radius disk.
    ``mid256``: 128 stations in a 1 km core plus 128 at log-spaced radii 1-8 km.
    ``wide512``: 256 stations in a 1 km dense core plus 256 at log-spaced radii 1-40 km.
    ``heights`` adds the Earth-curvature sagitta -r^2/(2 R) plus N(0, 10 m) jitter.
    """
    if kind == "disk128":
        en = _disk(rng, 128, 1500.0)
    elif kind == "mid256":
        en = np.concatenate([_disk(rng, 128, 1000.0), _log_arms(rng, 128, 1000.0, 8000.0)])
    elif kind == "wide512":
        en = np.concatenate([_disk(rng, 256, 1000.0), _log_arms(rng, 256, 1000.0, 40000.0)])
    else:
        raise ValueError(f"unknown station layout {kind!r}")
    up = np.zeros(len(en))
    if heights:
        r2 = (en ** 2).sum(axis=1)
        up = -r2 / (2 * EARTH_RADIUS) + rng.normal(0.0, 10.0, len(en))
    return np.concatenate([en, up[:, None]], axis=1)


def baseline_uvw(enu: np.ndarray, hour_angle: float, declination: float,
                 latitude: float = SITE_LATITUDE) -> np.ndarray:
    """uvw (metres) of all station pairs i < j, row order (0,1), (0,2), ..., (n-2, n-1)."""
    e, n, u = enu[:, 0], enu[:, 1], enu[:, 2]
    x = -math.sin(latitude) * n + math.cos(latitude) * u
    y = e
    z = math.cos(latitude) * n + math.sin(latitude) * u
    xyz = np.stack([x, y, z], axis=1)
    i, j = np.triu_indices(len(enu), k=1)
    L = xyz[j] - xyz[i]
    sh, ch = math.sin(hour_angle), math.cos(hour_angle)
    sd, cd = math.sin(declination), math.cos(declination)
    uu = sh * L[:, 0] + ch * L[:, 1]
    vv = -sd * ch * L[:, 0] + sd * sh * L[:, 1] + cd * L[:, 2]
    ww = cd * ch * L[:, 0] - cd * sh * L[:, 1] + sd * L[:, 2]
    return np.stack([uu, vv, ww], axis=1)


def point_sources(rng, n, flux_lo, flux_hi, field):
    flux = np.exp(rng.uniform(np.log(flux_lo), np.log(flux_hi), n))
    lm = rng.uniform(-field / 2, field / 2, (n, 2))
    return np.concatenate([flux[:, None], lm], axis=1)


def sky_visibilities(uvw_m: np.ndarray, freqs_hz: np.ndarray, sources: np.ndarray,
                     chunk_rows: int = 16384, device: Optional[str] = None) -> np.ndarray:
    """Noise-free visibilities [num_rows, num_channels] complex128 of a point-source sky.

    V(row, chan) = sum_s S_s exp(-2 pi i (f/c) (u l + v m + w (n - 1))), evaluated in FP64 with
    torch (on the GPU when one is present, else on all host cores). Channels are advanced by a
    phasor recurrence per channel step, re-anchored by a direct exponential every 16 channels.
    """
    import torch

    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    nr, nc = uvw_m.shape[0], len(freqs_hz)
    out = np.zeros((nr, nc), dtype=np.complex128)
    src = torch.as_tensor(sources, dtype=torch.float64, device=device)
    S = src[:, 0].to(torch.complex128)
    l, m = src[:, 1], src[:, 2]
    nn = torch.sqrt(1.0 - l * l - m * m) - 1.0
    f = np.asarray(freqs_hz, dtype=np.float64) / C_LIGHT
    for r0 in range(0, nr, chunk_rows):
        blk = torch.as_tensor(uvw_m[r0:r0 + chunk_rows], dtype=torch.float64, device=device)
        phi = -2 * math.pi * (torch.outer(blk[:, 0], l) + torch.outer(blk[:, 1], m)
                              + torch.outer(blk[:, 2], nn))
        res = torch.empty((blk.shape[0], nc), dtype=torch.complex128, device=device)
        z = step = None
        for c in range(nc):
            if c % 16 == 0:
                z = torch.polar(torch.ones_like(phi), phi * f[c])
                if c + 1 < nc:
                    step = torch.polar(torch.ones_like(phi), phi * (f[c + 1] - f[c]))
            else:
                z = z * step
            res[:, c] = z @ S
        out[r0:r0 + chunk_rows] = res.cpu().numpy()
    return out


# ------------------------------------------------------------------------------------------
# configurations
# ------------------------------------------------------------------------------------------
CONFIGS = {
    # name: (index, layout, nchan, f_lo, f_hi, N, cell, dec_deg, field, faint_sources, heights)
    "small": (0, "disk128", 16, 140e6, 155e6, 256, 4e-4, -30.0, 0.1, 0, False),
    "precision": (1, "wide512", 64, 140e6, 170e6, 2048, 5e-5, -30.0, 0.1, 200, False),
    "batching": (2, "mid256", 64, 140e6, 170e6, 1024, 1e-4, -30.0, 0.1, 0, False),
    "widefield": (3, "wide512", 64, 140e6, 170e6, 4096, 0.3 / 4096, 30.0, 0.3, 0, True),
}


def make_snapshot(config: str = "small", *, hour_angle: float = 0.0, nchan: Optional[int] = None,
                  flag_fraction_rows: float = 0.05, flag_fraction_samples: float = 0.0,
                  snapshot_index: int = 0, layout: Optional[str] = None,
                  image_size: Optional[int] = None, cell_size: Optional[float] = None,
                  n_rows_limit: Optional[int] = None) -> Snapshot:
    """Build one synthetic snapshot of a named configuration (seeded, deterministic)."""
    idx, lay, nch, flo, fhi, N, cell, dec, field, nfaint, heights = CONFIGS[config]
    lay = layout or lay
    nch = nchan or nch
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + idx))
    enu = station_layout(lay, rng, heights=heights)
    sources = point_sources(rng, 20, 0.1, 10.0, field)
    if nfaint:
        sources = np.concatenate([sources, point_sources(rng, nfaint, 1e-3, 1e-2, field)])
    # per-snapshot stream: independent of the layout stream
    srng = np.random.Generator(np.random.PCG64([SEED_BASE + idx, snapshot_index]))
    uvw = baseline_uvw(enu, hour_angle, math.radians(dec))
    if n_rows_limit is not None:
        uvw = uvw[:n_rows_limit]
    freqs = np.linspace(flo, fhi, nch)
    vis = sky_visibilities(uvw, freqs, sources)        # [rows, chan]
    nr = uvw.shape[0]
    sig = 0.05 / math.sqrt(2.0)
    noise = srng.standard_normal((4, nr, nch)) * sig
    v0 = (vis + noise[0] + 1j * noise[1])
    v3 = (vis + noise[2] + 1j * noise[3])
    w = srng.uniform(0.5, 1.0, (2, nr, nch))
    flags = np.zeros((2, nr, nch), dtype=bool)
    if flag_fraction_rows > 0:
        rows = srng.random(nr) < flag_fraction_rows
        flags[:, rows, :] = True
    if flag_fraction_samples > 0:
        fs = srng.random((nr, nch)) < flag_fraction_samples
        flags[:, fs] = True

    def flat(a):  # [rows, chan] -> channel-major flat
        return np.ascontiguousarray(a.T).reshape(-1)

    return Snapshot(
        num_rows=nr, num_channels=nch,
        uvw=uvw.astype(np.float32), frequencies_hz=freqs.astype(np.float32),
        vis0_real=flat(v0.real).astype(np.float32), vis0_imag=flat(v0.imag).astype(np.float32),
        vis3_real=flat(v3.real).astype(np.float32), vis3_imag=flat(v3.imag).astype(np.float32),
        flag0=flat(flags[0]).astype(np.uint8), flag3=flat(flags[1]).astype(np.uint8),
        weight0=flat(w[0]).astype(np.float32), weight3=flat(w[1]).astype(np.float32),
        array_center_x=float(np.float32(ARRAY_CENTER[0])),
        image_size=image_size or N, cell_size=cell_size or cell,
        time=float(snapshot_index), sources=sources, uvw64=uvw)


def batching_stream(n_snapshots: int = 256, *, seed_offset: int = 0,
                    n_rows_limit: Optional[int] = None) -> List[Snapshot]:
    """The batching configuration: hour angles spread over +-3 h, channel counts drawn from
    {16, 32, 64}, sample-level flag fractions uniform in 0-40 %."""
    rng = np.random.Generator(np.random.PCG64(SEED_BASE + 2 + 1000 * (1 + seed_offset)))
    has = np.linspace(-3.0, 3.0, n_snapshots) * (math.pi / 12.0)
    out = []
    for i in range(n_snapshots):
        nch = int(rng.choice([16, 32, 64]))
        ff = float(rng.uniform(0.0, 0.4))
        out.append(make_snapshot("batching", hour_angle=float(has[i]), nchan=nch,
                                 flag_fraction_rows=0.0, flag_fraction_samples=ff,
                                 snapshot_index=i + 1, n_rows_limit=n_rows_limit))
    return out
