"""Plan speculation in the engine.

A call with the same shape as the engine's previous call (image size, cell, rows, samples) does not
wait for its w statistics before gridding: it launches with the previous call's slab and Chebyshev
counts, takes the slab geometry and 1 / |det| from a device-side plan computed from its own
statistics, and checks the counts against its host decision afterwards, imaging again when they
differ. Every image must equal a fresh engine's image of the same snapshot (relative RMS < 1e-6, the
order of floating-point atomic adds), with the same slab configuration bit for bit."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from svdimager_b200 import api, synth

pytestmark = pytest.mark.gpu

OPTS = dict(edge_mode=api.EDGE_STRICT, k_rule=api.KRULE_TARGET, target_error=1e-6)
KEYS = ("num_slabs", "num_terms", "slab_r3_min", "slab_width", "slab_half", "num_gridded", "vin")


def _fresh(s, **kw):
    with api.Engine(**kw) as e:
        img = e.image(s)
        return img, e.stats()


def test_same_and_changed_counts_match_fresh_engines(cuda_device):
    a = synth.make_snapshot("small", snapshot_index=0)
    b = synth.make_snapshot("small", snapshot_index=1)  # same baselines, other noise and flags
    uvw = a.uvw.copy()
    uvw[:, 2] += np.float32(0.3) * uvw[:, 0]            # a wide w range: more slabs or terms
    c = dataclasses.replace(a, uvw=uvw)
    refs = {k: _fresh(s, **OPTS) for k, s in (("a", a), ("b", b), ("c", c))}
    assert refs["c"][1]["num_planes"] != refs["a"][1]["num_planes"]
    assert refs["b"][1]["num_planes"] == refs["a"][1]["num_planes"]
    with api.Engine(**OPTS) as e:
        for name, s in (("a", a), ("a", a), ("b", b), ("c", c), ("c", c), ("a", a)):
            img = e.image(s)
            st = e.stats()
            ref, rst = refs[name]
            for k in KEYS:
                assert st[k] == rst[k], (name, k)
            assert O.rel_rms(img, ref) < 1e-6, name


def test_archive_entry_repeats_match_a_fresh_engine(cuda_device):
    from tests.golden.make_golden import quartet
    visr, visi, b, v, N, cell = quartet()
    with api.Engine(api.archive_options()) as e:
        ref = e.fipipe(visr, visi, b, v, N, cell)
        rst = e.stats()
    with api.Engine(api.archive_options()) as e:
        for _ in range(3):
            img = e.fipipe(visr, visi, b, v, N, cell)
            st = e.stats()
            for k in KEYS:
                assert st[k] == rst[k], k
            assert O.rel_rms(img, ref) < 1e-6
