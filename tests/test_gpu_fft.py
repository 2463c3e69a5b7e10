"""The pruned inverse FFT against numpy: the moment planes after the FFT (BUF_MOMENTS) equal the
unnormalised inverse 2-D DFT of the gridded planes (BUF_GRID) on the N columns the recombination
reads, for the grid sizes of the shared-memory column transform (G = 2^a and 3 * 2^a up to 1536
and from 4096: radix-3, -16 and -2/4/8 passes), of the strided cuFFT column plan (G = 150, 2048,
3072) and of the full 2-D plan (G = 383, prime); odd N puts the read columns at an odd start and leaves the
last column block short. FP32 transforms: 2e-6 relative L2."""
import numpy as np
import pytest

from svdimager_b200 import api, synth

pytestmark = pytest.mark.gpu

FFT_TOL = 2e-6


def _planes(N, cell, sigma=1.5, nchan=8, rows=3000, **kw):
    s = synth.make_snapshot("small", n_rows_limit=rows, nchan=nchan)
    with api.Engine(keep_grid=1, sigma=sigma, k_rule=api.KRULE_FIXED, fixed_k=1, **kw) as e:
        e.image(s, N, cell)
        st = e.stats()
        G = st["grid_size"]
        grid = e.buffer(api.BUF_GRID).reshape(-1, G, G)
        mom = e.buffer(api.BUF_MOMENTS).reshape(-1, G, G)
    return G, grid, mom


@pytest.mark.parametrize("N,sigma,G_expect", [
    (64, 1.5, 96), (128, 1.5, 192), (256, 1.5, 384), (512, 1.5, 768), (1024, 1.5, 1536),
    (2048, 1.5, 3072), (64, 2.0, 128), (256, 2.0, 512), (1024, 2.0, 2048), (2048, 2.0, 4096),
    (100, 1.5, 150), (255, 1.5, 383),
    # odd N: the read columns start at an odd column (8-byte copies) and the last block is ragged
    (47, 2.0, 96), (95, 2.0, 192)])
def test_moments_are_the_inverse_dft_of_the_grid(cuda_device, N, sigma, G_expect):
    G, grid, mom = _planes(N, 4e-4 * 256 / N, sigma=sigma)
    assert G == G_expect
    c0 = G // 2 - N // 2
    ref = np.fft.ifft2(grid.astype(np.complex128), axes=(1, 2)) * (G * G)
    got = mom[:, :, c0:c0 + N].astype(np.complex128)
    want = ref[:, :, c0:c0 + N]
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    print("G", G, "rel L2", err)
    assert err < FFT_TOL


def test_wide_grid_moments(cuda_device):
    """The wide-field grid: 4096^2 at sigma 1.5 gives G = 6144 (four columns per CTA, 192 KB of
    shared memory), checked on a random subset of columns against a numpy transform of those
    columns."""
    N = 4096
    G, grid, mom = _planes(N, 5e-5, rows=2000, nchan=4)
    assert G == 6144
    c0 = G // 2 - N // 2
    rows_done = np.fft.ifft(grid[0].astype(np.complex128), axis=1) * G  # the row pass
    rng = np.random.default_rng(3)
    cols = c0 + rng.choice(N, 64, replace=False)
    want = np.fft.ifft(rows_done[:, cols], axis=0) * G
    got = mom[0][:, cols].astype(np.complex128)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    print("G", G, "rel L2", err)
    assert err < FFT_TOL
