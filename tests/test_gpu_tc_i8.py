"""Parity of the exact integer tensor-core gridder (tcgen05.mma kind::i8: 22-bit fixed-point row
weights and column weights x visibility as three byte digits, int32 accumulation in tensor memory)
with the oracle, with the FP32 gridder and with the FP64 direct DFT.

The integer path grids one Chebyshev term per launch (T_n(s) folded into the sample's value), so
most tests fix K = 1 on both sides and the multi-term tests compare every moment plane of K = 8 and
of a multi-slab w-term case. Tile binning (24 x 8 tiles) stays bit-exact. Grid planes: each contribution is quantised to 2^-22
of the row weight's range and of the key's largest |value| (the sums themselves are exact), plus
the ES polynomial (<= 1.2e-7); planes are compared at I8_GRID_TOL relative L2. Images: 1e-5
relative RMS, as for the FP32 path."""
import numpy as np
import pytest

from oracle import oracle as O
from svdimager_b200 import api, synth
from tests.conftest import snapshot
from tests.test_gpu_parity import IMG_TOL, _check_binning, _scale, _slab_config_from_stats, _tilted_basis

pytestmark = pytest.mark.gpu

I8_GRID_TOL = 4e-6


def _i8(**kw):
    base = dict(gridder=api.GRIDDER_TC_I8, k_rule=api.KRULE_FIXED, fixed_k=1)
    base.update(kw)
    return base


@pytest.fixture(scope="module")
def i8_run(cuda_device, small_snapshot):
    s = small_snapshot
    e = api.Engine(**_i8(keep_grid=1))
    img = e.image(s)
    st = e.stats()
    return dict(engine=e, image=img, stats=st, snap=s)


def test_i8_path_is_used(i8_run):
    st = i8_run["stats"]
    assert st["used_tc"] == 1
    assert st["tile"] == 24 and st["tile_cols"] == 8
    assert st["num_terms"] == 1


def test_i8_tile_binning_bit_exact(i8_run):
    s, e, st = i8_run["snap"], i8_run["engine"], i8_run["stats"]
    r = O.expand_coords(e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S))
    _check_binning(e, st, r, e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG), s.cell_size)


def test_i8_grid_planes_match_oracle(i8_run):
    s, e, st = i8_run["snap"], i8_run["engine"], i8_run["stats"]
    G = st["grid_size"]
    r = O.expand_coords(e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S))
    vin = np.array(st["vin"]).reshape(3, 3)
    inv_det = 1.0 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    sc = _slab_config_from_stats(st)
    og = O.grid(r, e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG), _scale(s.cell_size, G), G, sc,
                inv_det)
    grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
    assert grid.shape == og.shape
    for p in range(og.shape[0]):
        den = np.linalg.norm(og[p])
        if den > 0:
            err = np.linalg.norm(grid[p] - og[p]) / den
            print("plane", p, "rel L2 vs oracle", err)
            assert err < I8_GRID_TOL, (p, err)
        # cells no footprint reaches stay exactly zero
        assert np.all(grid[p][og[p] == 0] == 0)


def test_i8_image_matches_oracle_and_fp32_path(i8_run):
    s = i8_run["snap"]
    o = O.image_sii(s, k_rule=1)
    assert i8_run["stats"]["num_slabs"] == o.sc.num_slabs
    assert O.rel_rms(i8_run["image"], o.image) < IMG_TOL
    with api.Engine(k_rule=api.KRULE_FIXED, fixed_k=1) as e:
        img32 = e.image(s)
        assert e.stats()["used_tc"] == 0
    assert O.rel_rms(i8_run["image"], img32) < IMG_TOL


def test_i8_edge_clipping_and_integer_positions(cuda_device):
    """Footprints clipped at the grid edge and exact-integer positions (the direct path with exact
    ES weights) against the oracle grid."""
    N, cell = 64, 2e-3
    G = 96
    scale = float(np.float32(cell)) * G
    rng = np.random.default_rng(5)
    n = 3000
    b = rng.uniform(-1.0, 1.0, (n, 3)) * (G / 2 + 3) / scale
    b[:, 2] *= 1e-3
    ints = rng.integers(-G // 2 + 5, G // 2 - 5, (300, 2)).astype(np.float64)
    b[:300, :2] = ints / scale
    b[300:400, 0] = ints[:100, 0] / scale
    b[400:500, 1] = ints[100:200, 1] / scale
    b = b.astype(np.float32)
    visr = rng.normal(size=n).astype(np.float32)
    visi = rng.normal(size=n).astype(np.float32)
    v = np.eye(3, dtype=np.float32)
    v[0] = [0.8, 0.6, 0.0]
    v[1] = [-0.6, 0.8, 0.0]
    with api.Engine(api.archive_options(**_i8(coord_mode=api.COORD_REF32, keep_grid=1))) as e:
        e.fipipe(visr, visi, b, v, N, cell)
        st = e.stats()
        assert st["used_tc"] == 1
        _check_binning(e, st, b.astype(np.float64), visr, visi, cell, coord_mode=1)
        grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
    inv_det = 1.0 / abs(0.8 * 0.8 + 0.6 * 0.6)
    og = O.grid(b.astype(np.float64), visr, visi, scale, G, _slab_config_from_stats(st), inv_det, coord_mode=1)
    assert np.linalg.norm(grid - og) / np.linalg.norm(og) < I8_GRID_TOL


def test_i8_pile_longer_than_one_accumulator_interval(cuda_device):
    """80,000 coincident samples with near-maximal, nearly equal values in one tile key: more than
    the 2048 K-blocks (65,536 samples) an int32 accumulator could hold, so the key's accumulation
    must be split (the gridder ends every interval with its 64-K-block chunk); every digit product of
    the pile is the same, the case that would overflow int32 first. Grid and image against the
    oracle."""
    N, cell, G = 64, 2e-3, 96
    scale = float(np.float32(cell)) * G
    rng = np.random.default_rng(13)
    n_pile, n_rest = 80_000, 5_000
    b = np.empty((n_pile + n_rest, 3))
    b[:n_pile] = np.array([5.29, -9.83, 0.0]) / scale
    b[n_pile:] = rng.uniform(-1.0, 1.0, (n_rest, 3)) * (G / 2 - 6) / scale
    b[:, 2] = rng.uniform(-1e-3, 1e-3, n_pile + n_rest)
    visr = np.concatenate([np.full(n_pile, 1.0e3), rng.normal(size=n_rest)]).astype(np.float32)
    visi = np.concatenate([np.full(n_pile, -999.0), rng.normal(size=n_rest)]).astype(np.float32)
    b = b.astype(np.float32)
    v = _tilted_basis()
    with api.Engine(api.archive_options(gridder=api.GRIDDER_TC_I8, coord_mode=api.COORD_REF32, keep_grid=1)) as e:
        img = e.fipipe(visr, visi, b, v, N, cell)
        st = e.stats()
        assert st["used_tc"] == 1  # the archive rule picks one Chebyshev term for |w| <= 1e-3
        grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
    o = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=1)
    V = v.astype(np.float64)
    inv_det = 1.0 / abs(V[0, 0] * V[1, 1] - V[0, 1] * V[1, 0])
    og = O.grid(b.astype(np.float64), visr, visi, scale, G, o.sc, inv_det, coord_mode=1)
    err = np.linalg.norm(grid - og) / np.linalg.norm(og)
    print("pile: grid rel L2 vs oracle", err, "image", O.rel_rms(img, o.image))
    assert err < I8_GRID_TOL
    assert O.rel_rms(img, o.image) < IMG_TOL


@pytest.mark.parametrize("N", [255, 100])
def test_i8_odd_and_small_image_sizes(cuda_device, N):
    s = synth.make_snapshot("small", n_rows_limit=3000, nchan=8)
    cell = 4e-4 * 256 / N
    with api.Engine(**_i8()) as e:
        img = e.image(s, N, cell)
        assert e.stats()["used_tc"] == 1
    o = O.image_sii(s, N, cell, k_rule=1)
    assert O.rel_rms(img, o.image) < IMG_TOL


def test_i8_repeat_calls_are_stable(cuda_device, small_snapshot):
    with api.Engine(**_i8()) as e:
        a = e.image(small_snapshot)
        b = e.image(small_snapshot)
    assert O.rel_rms(a, b) < 1e-6


def test_i8_precision_config_accuracy(cuda_device):
    """The headline configuration (8.4M samples, 2048^2, K = 1) on the integer tensor-core
    gridder: sample accounting, agreement with the FP32 gridder and accuracy against the FP64 DFT
    at random pixels (strict inclusion)."""
    s = snapshot("precision")
    kw = dict(edge_mode=api.EDGE_STRICT, presplat=1, k_rule=api.KRULE_TARGET, target_error=1e-6)
    with api.Engine(gridder=api.GRIDDER_TC_I8, **kw) as e:
        R = e.image(s)
        st = e.stats()
        vr, vi = e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG)
        q, sv = e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S)
    assert st["used_tc"] == 1 and st["num_terms"] == 1
    with api.Engine(**kw) as e:
        R32 = e.image(s)
    assert O.rel_rms(R, R32) < IMG_TOL
    vin = np.array(st["vin"]).reshape(3, 3)
    r = O.expand_coords(q, sv)
    G = st["grid_size"]
    inc = O.inclusion_mask(r, _scale(s.cell_size, G), G, edge_mode=1)
    assert st["num_gridded"] == int(inc.sum())
    rng = np.random.default_rng(7)
    N = s.image_size
    px, py = rng.integers(0, N, 256), rng.integers(0, N, 256)
    inv_det = 1 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    d = O.dft_pixels_sep(q, sv, vr, vi, inv_det, s.num_samples, vin, N, float(np.float32(s.cell_size)), px, py, inc)
    err = O.rel_rms(R[py, px], d)
    peak = np.max(np.abs(R[py, px] - d)) / np.max(np.abs(d))
    print("precision (integer tensor core): rel RMS vs FP64 DFT", err, "peak", peak, "vs FP32 path",
          O.rel_rms(R, R32))
    assert err < IMG_TOL


@pytest.fixture(scope="module")
def i8_multi_run(cuda_device, small_snapshot):
    """The main path's default Chebyshev rule (K = 8 on this snapshot) on the integer gridder."""
    s = small_snapshot
    e = api.Engine(gridder=api.GRIDDER_TC_I8, keep_grid=1)
    img = e.image(s)
    return dict(engine=e, image=img, stats=e.stats(), snap=s)


def test_i8_multi_term_planes_match_oracle(i8_multi_run):
    """Every one of the K = 8 moment planes (one launch per term, T_n(s) folded into B) against the
    oracle grid, each relative to its own norm."""
    s, e, st = i8_multi_run["snap"], i8_multi_run["engine"], i8_multi_run["stats"]
    assert st["used_tc"] == 1 and st["num_terms"] == 8
    assert st["tile"] == 24 and st["tile_cols"] == 8
    G = st["grid_size"]
    r = O.expand_coords(e.buffer(api.BUF_Q).reshape(-1, 3), e.buffer(api.BUF_S))
    vin = np.array(st["vin"]).reshape(3, 3)
    inv_det = 1.0 / abs(vin[0, 0] * vin[1, 1] - vin[0, 1] * vin[1, 0])
    og = O.grid(r, e.buffer(api.BUF_VIS_REAL), e.buffer(api.BUF_VIS_IMAG), _scale(s.cell_size, G), G,
                _slab_config_from_stats(st), inv_det)
    grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
    assert grid.shape == og.shape and og.shape[0] == 8
    for p in range(og.shape[0]):
        den = np.linalg.norm(og[p])
        assert den > 0
        err = np.linalg.norm(grid[p] - og[p]) / den
        print("term", p, "rel L2 vs oracle", err)
        assert err < I8_GRID_TOL, (p, err)


def test_i8_multi_term_image_matches_oracle_and_fp32_path(i8_multi_run):
    s = i8_multi_run["snap"]
    o = O.image_sii(s)
    assert o.sc.K == 8
    assert O.rel_rms(i8_multi_run["image"], o.image) < IMG_TOL
    with api.Engine() as e:
        img32 = e.image(s)
        assert e.stats()["used_tc"] == 0 and e.stats()["num_terms"] == 8
    assert O.rel_rms(i8_multi_run["image"], img32) < IMG_TOL


def test_i8_wterm_multi_slab_matches_oracle_and_dft(cuda_device):
    """Non-coplanar snapshot on the integer gridder: several w-slabs x 12 Chebyshev terms (twelve
    launches over the slabs' keys), against the oracle and the FP64 DFT."""
    s = snapshot("widefield", nchan=4, n_rows_limit=6000, image_size=128, cell_size=6e-4)
    with api.Engine(gridder=api.GRIDDER_TC_I8, k_rule=api.KRULE_FIXED, fixed_k=12, target_alpha=2.0,
                    edge_mode=api.EDGE_STRICT, presplat=1) as e:
        R = e.image(s)
        st = e.stats()
    o = O.image_sii(s, edge_mode=1, k_rule=12, target_alpha=2.0)
    assert st["used_tc"] == 1
    assert st["num_slabs"] == o.sc.num_slabs > 1 and st["num_terms"] == 12
    assert O.rel_rms(R, o.pre) < IMG_TOL
    rng = np.random.default_rng(2)
    N = s.image_size
    px, py = rng.integers(0, N, 300), rng.integers(0, N, 300)
    inc = O.inclusion_mask(o.r, _scale(s.cell_size, o.G), o.G, edge_mode=1)
    inv_det = 1 / abs(o.vin[0, 0] * o.vin[1, 1] - o.vin[0, 1] * o.vin[1, 0])
    d = O.dft_pixels(o.r, o.vr, o.vi, inv_det, s.num_samples, o.vin, N, float(np.float32(s.cell_size)), px, py,
                     inc)
    m = np.isfinite(d)
    assert O.rel_rms(R[py, px][m], d[m]) < IMG_TOL
