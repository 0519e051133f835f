"""The z-direction transform (semtex's dDFTr, femlib/fourier.c:47-171).

CPU: the oracle's direct-DFT restatement against a known answer (a single
cosine and sine mode), against an independent FFT-based computation of the
same packing, and for its own round trip.  GPU: sx_transform_z against the
oracle for even lengths with factors 2, 3, 5 and ragged point counts, and
the forward-inverse round trip in place -- the one-pass register kernels
(2, 4, ..., 64), the shared-memory kernels (128, 256, 512) and the cuFFT
path (other lengths).
"""
import numpy as np
import pytest

from oracle.oracle import transform_z as oracle_tz


def test_oracle_known_answer():
    nz, npts = 12, 5
    j = np.arange(nz)[:, None]
    x = 0.7 + 2.0 * np.cos(2 * np.pi * 3 * j / nz) + 0.5 * np.sin(2 * np.pi * 2 * j / nz) \
        + 0.25 * np.cos(np.pi * j) + np.zeros((nz, npts))
    X = oracle_tz(x, +1)
    want = np.zeros_like(X)
    want[0] = 0.7          # mode 0: the mean
    want[1] = 0.25         # Nyquist
    want[6] = 1.0          # Re X_3 = 2.0 / 2
    want[5] = -0.25        # Im X_2 = -0.5 / 2 (exp(-i...) convention)
    assert np.allclose(X, want, atol=1e-14)


@pytest.mark.parametrize("nz", [2, 4, 6, 10, 16, 30, 64])
def test_oracle_matches_fft_packing_and_round_trip(nz):
    rng = np.random.default_rng(nz)
    x = rng.standard_normal((nz, 37))
    X = oracle_tz(x, +1)
    F = np.fft.rfft(x, axis=0) / nz
    ref = np.empty_like(x)
    ref[0] = F[0].real
    ref[1] = F[nz // 2].real
    for k in range(1, nz // 2):
        ref[2 * k] = F[k].real
        ref[2 * k + 1] = F[k].imag
    assert np.allclose(X, ref, atol=1e-13)
    assert np.allclose(oracle_tz(X, -1), x, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("nz,npts,stride", [(2, 33, 34), (4, 130, 130), (8, 129, 132), (16, 82944, 82944),
                                            (32, 300, 300), (64, 4096, 4100), (64, 82944, 82944),
                                            (128, 999, 1000), (256, 2050, 2050), (256, 410240, 410240),
                                            (512, 100, 100), (6, 1000, 1000), (30, 257, 260),
                                            (96, 333, 340), (160, 70, 72)])
def test_transform_matches_oracle(nz, npts, stride):
    import torch
    import semtex_b200 as sx
    rng = np.random.default_rng(nz + npts)
    x = rng.standard_normal((nz, stride))
    d = torch.tensor(x, device="cuda")
    sx.transform_z(d.data_ptr(), nz, stride, npts, +1)
    X = d.cpu().numpy()
    Xo = oracle_tz(x[:, :npts], +1)
    err = np.abs(X[:, :npts] - Xo).max() / np.abs(Xo).max()
    assert err <= 1e-13, err
    assert np.array_equal(X[:, npts:], x[:, npts:])   # padding untouched
    sx.transform_z(d.data_ptr(), nz, stride, npts, -1)
    back = d.cpu().numpy()
    err = np.abs(back[:, :npts] - x[:, :npts]).max() / np.abs(x).max()
    assert err <= 1e-13, err


@pytest.mark.gpu
def test_transform_rejects_bad_lengths():
    import torch
    import semtex_b200 as sx
    d = torch.zeros((14, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(sx.SolverError):
        sx.transform_z(d.data_ptr(), 14, 8, 8, +1)      # prime factor 7
    with pytest.raises(sx.SolverError):
        sx.transform_z(d.data_ptr(), 9, 8, 8, +1)       # odd
    sx.transform_z(d.data_ptr(), 1, 8, 8, +1)           # nz = 1: nothing to do
