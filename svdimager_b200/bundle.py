"""Snapshot bundle: a single-file stand-in for a Measurement Set (casacore is not available).

It carries exactly the columns the reference's reader uses (SVDIntegratedImager.cu:180-378):
TIME, UVW, DATA, FLAG and WEIGHT_SPECTRUM of the main table, CHAN_FREQ of SPECTRAL_WINDOW and
ARRAY_CENTER of OBSERVATION. Layout (little-endian):

    char[8]  magic "SVDIMS01"
    uint64   num_rows, num_channels, num_pols, has_weight_spectrum
    double   array_center[3]
    double   TIME[num_rows]
    double   UVW[num_rows][3]
    double   CHAN_FREQ[num_channels]
    float    DATA[num_rows][num_channels][num_pols][2]      (re, im)
    uint8    FLAG[num_rows][num_channels][num_pols]
    float    WEIGHT_SPECTRUM[num_rows][num_channels][num_pols]  (if has_weight_spectrum)
"""
from __future__ import annotations

import struct
from typing import List, Sequence

import numpy as np

MAGIC = b"SVDIMS01"


def write_bundle(path: str, snapshots: Sequence, num_pols: int = 4):
    """Write snapshots (synth.Snapshot) as consecutive TIME groups of one bundle.
    All snapshots must share the channel set. Pols 1 and 2 are written as zeros."""
    C = snapshots[0].num_channels
    R = sum(s.num_rows for s in snapshots)
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<4Q", R, C, num_pols, 1))
        f.write(struct.pack("<3d", snapshots[0].array_center_x, 0.0, 0.0))
        f.write(np.concatenate([np.full(s.num_rows, s.time) for s in snapshots]).astype("<f8").tobytes())
        f.write(np.concatenate([s.uvw64 if s.uvw64 is not None else s.uvw for s in snapshots])
                .astype("<f8").tobytes())
        f.write(np.asarray(snapshots[0].frequencies_hz, np.float64).astype("<f8").tobytes())
        for part in ("data", "flag", "weight"):
            for s in snapshots:
                r, c = s.num_rows, s.num_channels

                def rc(a):  # channel-major flat -> [row][chan]
                    return np.asarray(a).reshape(c, r).T

                if part == "data":
                    d = np.zeros((r, c, num_pols, 2), np.float32)
                    d[:, :, 0, 0], d[:, :, 0, 1] = rc(s.vis0_real), rc(s.vis0_imag)
                    d[:, :, 3, 0], d[:, :, 3, 1] = rc(s.vis3_real), rc(s.vis3_imag)
                    f.write(d.astype("<f4").tobytes())
                elif part == "flag":
                    d = np.zeros((r, c, num_pols), np.uint8)
                    d[:, :, 0], d[:, :, 3] = rc(s.flag0), rc(s.flag3)
                    f.write(d.tobytes())
                else:
                    d = np.ones((r, c, num_pols), np.float32)
                    d[:, :, 0], d[:, :, 3] = rc(s.weight0), rc(s.weight3)
                    f.write(d.astype("<f4").tobytes())
