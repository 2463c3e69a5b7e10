"""Autotuner for the imaging options of a family of snapshots (same layout, image size and cell).

The reference fixes its kernel (support W = 8, beta = 15.3704 at oversampling 1.5,
SVDIntegratedImager.cu:884-888, 1510) and picks only the Chebyshev order. Here the gridder (FP32
CUDA-core or tensor-core), its tile size, the ES support W, the oversampling sigma (with the ES
beta that goes with W and sigma) and the Chebyshev error target are chosen per family: every
candidate images the representative snapshots once with presplat = 1 and is checked against the
library's FP64 direct DFT at random pixels (`Engine.dft_pixels`), then timed as one batch of those
snapshots (median of several graph launches); the fastest candidate whose relative RMS error stays
within the target wins. The Chebyshev order K and the
w-slab count follow from the error target per snapshot (k_rule TARGET: the fewest moment planes
that meet it)."""
from __future__ import annotations

import itertools
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import api

REF_BETA = 15.3704324328   # W = 8 at sigma = 1.5 (SVDIntegratedImager.cu:884-888)
SUPPORTS = (6, 8, 10, 12)
SIGMAS = (1.25, 1.5, 1.75, 2.0)


def es_beta(W: int, sigma: float) -> float:
    """ES beta for support W at oversampling sigma: the reference's beta at (8, 1.5) scaled by W
    and by the usable fraction of the kernel's spectrum, 1 - 1 / (2 sigma)."""
    return REF_BETA * (W / 8.0) * (1.0 - 1.0 / (2.0 * sigma)) / (1.0 - 1.0 / 3.0)


def candidates(supports: Sequence[int] = SUPPORTS, sigmas: Sequence[float] = SIGMAS,
               gridders: Sequence[str] = ("fp32", "tc"), tiles: Sequence[int] = (32, 64)) -> List[Dict]:
    """Option sets to try. The tensor-core gridder needs W <= 8 (and one moment plane per slab,
    which the engine checks per snapshot, falling back to the FP32 gridder otherwise)."""
    out = []
    for W, sg in itertools.product(supports, sigmas):
        base = dict(support=W, sigma=float(sg), beta=es_beta(W, sg))
        if "fp32" in gridders:
            for t in tiles:
                out.append(dict(base, gridder=api.GRIDDER_FP32, tile=t))
        if "tc" in gridders and W <= 8:
            out.append(dict(base, gridder=api.GRIDDER_TC, tile=0))
    return out


@dataclass
class Trial:
    options: Dict
    error: float = math.inf          # worst relative RMS over the representative snapshots
    ms: float = math.inf             # device time per snapshot in a batch of the snapshots
    num_terms: List[int] = field(default_factory=list)
    num_slabs: List[int] = field(default_factory=list)
    used_tc: bool = False
    failure: Optional[str] = None


def _rel_rms(a: np.ndarray, b: np.ndarray) -> float:
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.sqrt(np.sum((a[m] - b[m]) ** 2) / max(np.sum(b[m] ** 2), 1e-300)))


# The library's default options (the reference's kernel): the candidate a tuned choice must beat.
DEFAULT_CANDIDATE = dict(support=8, sigma=1.5, beta=REF_BETA, gridder=api.GRIDDER_FP32, tile=0)


def _batch_ms(snapshots, N: int, cell_size: float, out, options: Dict, repeats: int) -> float:
    """Device time per snapshot of `snapshots` imaged as one batch (the way batches run: every
    stage over all snapshots at once), median over `repeats` graph launches."""
    import torch
    imgs = out.new_zeros((len(snapshots), N, N))
    stream = torch.cuda.Stream(out.device)
    with api.Engine(**options) as e:
        b = api.Batch(e, snapshots, N, cell_size, imgs.data_ptr())
        try:
            b.launch(stream.cuda_stream)  # warm
            b.check()
            ms = []
            for _ in range(max(1, repeats)):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                b.launch(stream.cuda_stream)
                e1.record(stream)
                b.check()
                ms.append(e0.elapsed_time(e1) / len(snapshots))
        finally:
            b.close()
    return float(np.median(ms))


def tune(snapshots, image_size: int, cell_size: float, out, *, target: float = 1e-5,
         cheb_target: float = 1e-6, npix: int = 64, repeats: int = 3, device: int = 0,
         cands: Optional[List[Dict]] = None, seed: int = 11, stream_ptr: int = 0,
         margin: float = 0.03):
    """Pick imaging options for `snapshots` (device descriptors from api.device_ms) at N x N.

    out: a torch float32 CUDA tensor of N x N used as scratch output. Returns (best options dict,
    list of Trial). Options common to every candidate: strict edges, k_rule TARGET at
    cheb_target. Each accurate candidate is timed over `repeats` passes (median); the default
    options are always tried, and another candidate replaces them only when it is faster by more
    than `margin` (timing noise is a few per cent)."""
    rng = np.random.default_rng(seed)
    N = int(image_size)
    px = rng.integers(0, N, npix)
    py = rng.integers(0, N, npix)
    common = dict(device=device, edge_mode=api.EDGE_STRICT, k_rule=api.KRULE_TARGET, target_error=cheb_target)
    trials = []
    out_ptr = out.data_ptr()
    opts = list(cands if cands is not None else candidates())
    if not any(all(o.get(k) == v for k, v in DEFAULT_CANDIDATE.items()) for o in opts):
        opts.append(dict(DEFAULT_CANDIDATE))
    for opt in opts:
        t = Trial(options=dict(opt))
        try:
            with api.Engine(**common, presplat=1, **opt) as e:
                for d in snapshots:
                    e.image_device(d, N, cell_size, out_ptr, stream_ptr)
                    st = e.stats()
                    t.num_terms.append(st["num_terms"])
                    t.num_slabs.append(st["num_slabs"])
                    t.used_tc = t.used_tc or bool(st["used_tc"])
                    host = out.cpu().numpy()
                    ref = e.dft_pixels(px, py)
                    t.error = max(t.error if math.isfinite(t.error) else 0.0,
                                  _rel_rms(host[py, px].astype(np.float64), ref))
            if t.error <= target:
                t.ms = _batch_ms(snapshots, N, cell_size, out, dict(common, **opt), repeats)
        except api.SvdiError as ex:
            t.failure = ex.message
        trials.append(t)
    ok = [t for t in trials if t.error <= target and math.isfinite(t.ms)]
    if not ok:
        raise RuntimeError(f"no candidate reaches the accuracy target {target}")
    best = min(ok, key=lambda t: t.ms)
    dflt = [t for t in ok if all(t.options.get(k) == v for k, v in DEFAULT_CANDIDATE.items())]
    if dflt and best.ms > (1.0 - margin) * dflt[0].ms:
        best = dflt[0]
    return dict(common, **best.options), trials
