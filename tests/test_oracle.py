"""The oracle (CPU restatement of the reference path) checked on its own: against the FP64 direct
DFT, against independent numerics (numpy eigh, scipy Bessel, sklearn PCA as in
archive/SVD_MFS.py:59-106), and against the reference binary's golden output when present."""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import snapshot


def test_collapse_matches_reference_formula(small_snapshot):
    s = small_snapshot
    vr, vi = O.collapse(s)
    # SVD_MFS.py:74-90 / SVDIntegratedImager.cu:606-616 in float32 numpy
    w0 = np.where(s.flag0 != 0, np.float32(0), s.weight0).astype(np.float32)
    w3 = np.where(s.flag3 != 0, np.float32(0), s.weight3).astype(np.float32)
    ws = (w0 + w3).astype(np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        er = np.where(ws > 0, ((s.vis0_real * w0).astype(np.float32) + (s.vis3_real * w3).astype(np.float32)) / ws, 0)
        ei = np.where(ws > 0, ((s.vis0_imag * w0).astype(np.float32) + (s.vis3_imag * w3).astype(np.float32)) / ws, 0)
    assert np.array_equal(vr, er.astype(np.float32))
    assert np.array_equal(vi, ei.astype(np.float32))
    # flag mask: exactly the samples flagged on both pols are zero
    both = (s.flag0 != 0) & (s.flag3 != 0)
    assert np.all(vr[both] == 0) and np.all(vi[both] == 0)


def test_collapse_flagged_nan_follows_reference_arithmetic():
    """Non-finite data under a flag: the reference multiplies the flagged polarisation by its zero
    weight (SVDIntegratedImager.cu:606-612), so NaN or Inf data there still yield NaN whenever the
    other polarisation carries weight, and 0 only when both are flagged."""
    from types import SimpleNamespace
    nan, inf = np.float32(np.nan), np.float32(np.inf)
    f32 = lambda *x: np.array(x, np.float32)
    s = SimpleNamespace(
        num_samples=5,
        vis0_real=f32(nan, inf, 1.0, nan, 2.0), vis0_imag=f32(0.5, 0.5, nan, nan, 0.0),
        vis3_real=f32(3.0, 3.0, 3.0, nan, 4.0), vis3_imag=f32(1.0, 1.0, 1.0, nan, 0.0),
        flag0=np.array([1, 1, 0, 1, 0], np.uint8), flag3=np.array([0, 0, 0, 1, 0], np.uint8),
        weight0=f32(1, 1, 1, 1, 1), weight3=f32(1, 1, 1, 1, 1))
    vr, vi = O.collapse(s)
    assert np.isnan(vr[0]) and vi[0] == np.float32(1.0)    # NaN * 0 is NaN
    assert np.isnan(vr[1]) and vi[1] == np.float32(1.0)    # Inf * 0 is NaN
    assert vr[2] == np.float32(2.0) and np.isnan(vi[2])    # unflagged NaN propagates
    assert vr[3] == 0 and vi[3] == 0                       # both flagged: 0, whatever the data
    assert vr[4] == np.float32(3.0) and vi[4] == 0


def test_preprocess_against_numpy_and_pca(small_snapshot):
    s = small_snapshot
    vin, q, sv, ev = O.preprocess64(s)
    b = np.concatenate([s.uvw.astype(np.float64) * f for f in sv])  # channel-major rows
    m = b.mean(axis=0)
    cov = (b - m).T @ (b - m)
    w, v = np.linalg.eigh(cov)
    assert np.allclose(np.sort(ev), w, rtol=1e-10)
    for i, col in enumerate((2, 1, 0)):
        assert abs(abs(np.dot(vin[i], v[:, col])) - 1) < 1e-10
    # orientation rules
    assert vin[0, 0] >= 0
    assert vin[1, 1] * s.array_center_x >= 0
    assert np.allclose(np.cross(vin[0], vin[1]), vin[2], atol=1e-12)
    # sklearn PCA as in SVD_MFS.py: Bin = transform(D) + M V^T equals the un-centred projection
    from sklearn.decomposition import PCA
    pca = PCA(3).fit(b)
    comp = pca.components_
    sign = np.sign(np.sum(comp * vin, axis=1))
    bin_mfs = pca.transform(b) + m @ comp.T
    r = O.expand_coords(q, sv)
    assert np.allclose(bin_mfs * sign, r, rtol=1e-9, atol=1e-6)


def test_bessel_against_scipy():
    from scipy.special import jv
    for x in (0.0, 1e-9, 1e-4, 0.3, 2.0, 9.7, 31.0, 57.0):
        j = np.zeros(40)
        O.lib().orc_bessel_j(x, 39, j.ctypes.data_as(O.ctypes.c_void_p))
        ref = jv(np.arange(40), x)
        assert np.allclose(j, ref, rtol=1e-11, atol=1e-15), x


def test_es_correction_matches_reference_quadrature():
    # The reference tabulates Phi with the 28-point Gauss-Legendre rule (positive half: 14 nodes,
    # the kernel sampled at the nodes, SVDIntegratedImager.cu:867-882); both approximate the same
    # integral, so they agree far below the 1e-5 image tolerance.
    N, G = 256, 384
    phi = O.es_correction(N, G)
    x, w = np.polynomial.legendre.leggauss(28)
    x, w = x[x > 0], w[x > 0]
    k = np.exp(O.REF_BETA * (np.sqrt(1 - x * x) - 1))
    i = np.arange(N // 2 + 1)
    ref = O.REF_SUPPORT * np.sum(k * w * np.cos(np.pi * (i[:, None] / G) * O.REF_SUPPORT * x), axis=1)
    assert np.max(np.abs(phi / ref - 1)) < 1e-6


def test_cheb_error_table_matches_direct_evaluation():
    from scipy.special import jv
    a = 7.3
    err = O.cheb_errors(a, 33, 257, 16)
    aa = np.linspace(0, a, 33)[:, None, None]
    s = np.linspace(-1, 1, 257)[None, :, None]
    n = np.arange(16)[None, None, :]
    T = np.cos(n * np.arccos(np.clip(s, -1, 1)))
    J = jv(n, aa)
    c = np.where(n == 0, 1.0, 2.0) * (1j ** n) * J * T
    approx = np.cumsum(c, axis=2)
    ex = np.exp(1j * aa * s)
    direct = np.max(np.abs(ex - approx), axis=(0, 1))
    assert np.allclose(err, direct, rtol=1e-8, atol=1e-14)


def test_oracle_gridding_matches_dft_small(small_snapshot):
    """Gridding + FFT + Chebyshev recombination + correction reproduces the direct FP64 DFT on the
    pixels it images (strict edge inclusion), to the ES kernel's accuracy."""
    s = small_snapshot
    img = O.image_sii(s, edge_mode=1)
    N = s.image_size
    rng = np.random.default_rng(1)
    px, py = rng.integers(0, N, 300), rng.integers(0, N, 300)
    scale = float(np.float32(s.cell_size)) * img.G
    inc = O.inclusion_mask(img.r, scale, img.G, edge_mode=1)
    inv_det = 1 / abs(img.vin[0, 0] * img.vin[1, 1] - img.vin[0, 1] * img.vin[1, 0])
    vin, q, sv, _ = O.preprocess64(s)
    d = O.dft_pixels_sep(q, sv, img.vr, img.vi, inv_det, s.num_samples, img.vin, N,
                         float(np.float32(s.cell_size)), px, py, inc)
    g = img.pre[py, px]
    assert O.rel_rms(g, d) < 3e-6


def test_dft_recurrence_matches_direct(small_snapshot):
    s = small_snapshot
    vin, q, sv, _ = O.preprocess64(s)
    vr, vi = O.collapse(s)
    r = O.expand_coords(q, sv)
    px, py = np.array([3, 100, 128, 200]), np.array([5, 128, 77, 250])
    a = O.dft_pixels(r, vr, vi, 1.0, s.num_samples, vin, s.image_size, s.cell_size, px, py)
    b = O.dft_pixels_sep(q, sv, vr, vi, 1.0, s.num_samples, vin, s.image_size, s.cell_size, px, py)
    assert np.allclose(a, b, rtol=1e-10)


def test_w_term_slabs_match_dft():
    """Non-coplanar snapshot (station heights): several w-slabs and Chebyshev terms reproduce the
    DFT including the w phase."""
    s = snapshot("widefield", nchan=4, n_rows_limit=6000, image_size=128, cell_size=6e-4)
    img = O.image_sii(s, edge_mode=1, k_rule=12, target_alpha=2.0)
    assert img.sc.num_slabs > 1 and img.sc.alpha_max > 2.0
    N = s.image_size
    rng = np.random.default_rng(2)
    px, py = rng.integers(0, N, 200), rng.integers(0, N, 200)
    scale = float(np.float32(s.cell_size)) * img.G
    inc = O.inclusion_mask(img.r, scale, img.G, edge_mode=1)
    inv_det = 1 / abs(img.vin[0, 0] * img.vin[1, 1] - img.vin[0, 1] * img.vin[1, 0])
    d = O.dft_pixels(img.r, img.vr, img.vi, inv_det, s.num_samples, img.vin, N,
                     float(np.float32(s.cell_size)), px, py, inc)
    g = img.pre[py, px]
    m = np.isfinite(d)
    assert O.rel_rms(g[m], d[m]) < 1e-5


def test_reprojection_variants_agree_for_small_fields(small_snapshot):
    """The simplified SIN deprojection (SVDIntegratedImager.cu:1338-1379) and the trigonometric one
    (archive/FIPkernels.cu:577-624) are the same projection for fields well inside the sphere."""
    s = small_snapshot
    img = O.image_sii(s)
    a = O.reproject(img.pre, s.image_size, float(np.float32(s.cell_size)), img.vin, "sii")
    b = O.reproject(img.pre, s.image_size, float(np.float32(s.cell_size)), img.vin, "fipk")
    assert O.rel_rms(a, b) < 1e-9


GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fipk_small.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="golden output of the reference binary absent")
def test_oracle_matches_reference_binary_golden():
    """Pins the oracle: the archive FIpipe of the reference, compiled unmodified for sm_100a and run
    on a B200 (tests/golden/make_golden.py), against the oracle's archive restatement with the
    reference's FP32 coordinate rounding."""
    from tests.golden.make_golden import digest, quartet
    z = np.load(GOLDEN)
    visr, visi, b, v, N, cell = quartet()
    assert str(z["input_sha256"]) == digest(visr, visi, b, v)
    img = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=1)
    # At cell 4e-4 rad the reference's reprojection (FP32, degrees, theta ~ 87 deg where one ulp
    # is 7.6e-6 deg) moves splat positions by ~3e-4 pixel, so its image carries ~3e-4 relative
    # rounding noise; the FP64 restatement agrees with both of its builds at that level.
    assert O.rel_rms(img.image, z["image_precise"]) < 1e-3
    assert O.rel_rms(img.image, z["image"]) < 1e-3
    assert int(z["K"]) == img.sc.K


GOLDEN_WIDE = os.path.join(os.path.dirname(__file__), "golden", "fipk_widecell.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN_WIDE), reason="golden output of the reference binary absent")
def test_oracle_matches_reference_binary_golden_wide_cell():
    """Pins the oracle at 1e-5: at cell 8e-3 rad the reference's FP32 reprojection noise is
    negligible, so the reference binary (IEEE-math build) and the restatement agree over the
    whole archive path (gridding, FFT, recombination, correction, reprojection, splat)."""
    from tests.golden.make_golden import digest, wide_cell_quartet
    z = np.load(GOLDEN_WIDE)
    visr, visi, b, v, N, cell = wide_cell_quartet()
    assert str(z["input_sha256"]) == digest(visr, visi, b, v)
    img = O.image_fipk(visr, visi, b, v, N, cell, coord_mode=1)
    assert O.rel_rms(img.image, z["image_precise"]) < 1e-5
    assert O.rel_rms(img.image, z["image"]) < 1e-4
    assert int(z["K"]) == img.sc.K


def _contract_key(p1, p2, G, W, T, edge_mode):
    """Binning contract for one sample at grid position (p1, p2), exact rational arithmetic:
    Q = floor(p 2^24), cell = Q >> 24, footprint [cell - (W/2 - 1), cell + W/2] (one cell wider
    on the low side when the position is an exact integer), clipped to [-G/2, (G-1)/2] or dropped
    (strict); tile = (low end - gmin) // T; record coordinate Q - tile origin 2^24."""
    from fractions import Fraction
    gmin, gmax, hw = -(G // 2), (G - 1) // 2, W // 2
    ntile = (G + T - 1) // T
    tiles, qrel = [], []
    for p in (p1, p2):
        if not abs(p) < 1e9:
            return -1, None
        Q = math.floor(Fraction(p) * 2**24)
        cell, frac = Q >> 24, Q & 0xFFFFFF
        lo, hi = (cell - (hw - 1) if frac else cell - hw), cell + hw
        if edge_mode == 1 and (lo < gmin or hi > gmax):
            return -1, None
        lo, hi = max(lo, gmin), min(hi, gmax)
        if lo > hi:
            return -1, None
        t = (lo - gmin) // T
        tiles.append(t)
        qrel.append(Q - (gmin + t * T) * 2**24)
    return tiles[0] * ntile + tiles[1], qrel


@pytest.mark.parametrize("edge_mode", [0, 1])
def test_tile_keys_contract_at_edge_positions(edge_mode):
    """The oracle's tile keys and record coordinates against an exact restatement of the binning
    contract at the positions where a floating-point split could go wrong: exact integers, values
    an ulp either side of them, tiny negatives, tile boundaries, both grid edges, and positions far
    off the grid. The device rule (one round-down conversion of p 2^24 to a 64-bit integer) is the
    same integer arithmetic; the GPU parity tests compare its records with these bit for bit."""
    G, W, T = 384, 8, 64
    gmin, gmax = -(G // 2), (G - 1) // 2
    pts = [0.0, -0.0, 1.0, -1.0, 0.5, -0.5, 5e-300, -5e-300, 1e-12, -1e-12, 3.0 - 2**-40, 3.0 + 2**-40,
           -3.0 - 2**-40, -3.0 + 2**-40, 2**-24, -(2**-24), 2**-25, -(2**-25)]
    for b in range(gmin, gmax + 1, T):   # tile boundaries of the footprint's low end (lo = p - 3)
        pts += [b + 3.0, b + 3.0 - 2**-30, b + 3.0 + 2**-30, b + 4.0 - 2**-30]
    for e in (gmin, gmax):                # both grid edges under clipping and strict rules
        pts += [e - 4.5, e - 4.0, e - 3.0, e - 0.25, e, e + 0.25, e + 3.0, e + 4.0, e + 4.5]
    pts += [1e9, -1e9, 2e9, 1e15, float("inf"), float("-inf"), float("nan")]
    rng = np.random.default_rng(7)
    pts += list(rng.uniform(gmin - 8, gmax + 8, 64))
    pts = np.array(pts, np.float64)
    p1, p2 = np.repeat(pts, len(pts)), np.tile(pts, len(pts))
    r = np.stack([p1, p2, np.zeros_like(p1)], axis=1)
    sc = O.SlabConfig(0.0, 1.0, 0.0, 0.0, 1, 1.0, 0.5, 2.0, 0.0, 1)
    keys, xq, yq, _ = O.tile_keys(r, 1.0, G, W, T, edge_mode, sc, records=True)
    n_kept = 0
    for k in range(len(p1)):
        key, q = _contract_key(float(p1[k]), float(p2[k]), G, W, T, edge_mode)
        assert keys[k] == key, (p1[k], p2[k], keys[k], key)
        if key >= 0:
            n_kept += 1
            assert (int(xq[k]), int(yq[k])) == (q[0], q[1]), (p1[k], p2[k])
    assert n_kept > len(p1) // 4


@pytest.mark.parametrize("N,cell,tilt", [(256, 4e-4, 0.0), (255, 4e-4, 0.3), (512, 3e-3, -0.8), (64, 2e-2, 1.2)])
def test_t3_statistics_against_numpy(N, cell, tilt):
    """max |t3| and the valid-pixel count over the rotated-frame pixels (SII:1029-1077, pixel
    offsets from the imaging kernel's integer centre), against a vectorised numpy restatement; and
    max |t3| equals its value at the smallest or largest valid radicand, since t3 is monotone in it."""
    c, s = math.cos(tilt), math.sin(tilt)
    vin = np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
    m, valid = O.t3_stats(vin, N, cell)
    y, x = np.mgrid[0:N, 0:N]
    t1, t2 = cell * (y - N // 2), cell * (x - N // 2)
    v13, v23, v33 = vin[0, 2], vin[1, 2], vin[2, 2]
    ra = 1.0 - (t1 + v13) ** 2 - (t2 + v23) ** 2
    ok = ra >= 0
    t3 = -v33 + (1.0 if v33 >= 0 else -1.0) * np.sqrt(ra[ok])
    assert valid == int(ok.sum()) > 0
    assert abs(m - np.abs(t3).max()) <= 1e-15 * max(1.0, m)
    ends = [ra[ok].min(), ra[ok].max()]
    at_ends = max(abs(-v33 + (1.0 if v33 >= 0 else -1.0) * math.sqrt(r)) for r in ends)
    assert abs(m - at_ends) <= 1e-15 * max(1.0, m)
