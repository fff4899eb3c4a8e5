"""Oracle transforms pinned to their published definitions (CPU only).

The reference calls FFTW 3.3.2 (makefile:141), which is absent here; its
transforms are pinned through numpy.fft / scipy.fft, which compute the same
definitions: r2c/c2r (ffts.f90:27-67, scalings ffts.f90:51,91-92) and
REDFT10/REDFT01 (ffts.f90:147-181, scalings ffts.f90:132-133,166,171).
"""
import numpy as np
import pytest
import scipy.fft as sfft

from oracle import pyoracle

D = pyoracle.dptr


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12, 15, 16, 60, 64, 96, 128, 256, 384, 1024, 7 * 9])
@pytest.mark.parametrize("sign", [-1, 1])
def test_complex_fft(n, sign):
    L = pyoracle.lib()
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    h = L.orc_fft_create(n)
    inp = np.ascontiguousarray(np.stack([x.real, x.imag], -1).ravel())
    out = np.zeros(2 * n)
    L.orc_fft_exec(h, D(inp), D(out), sign)
    L.orc_fft_destroy(h)
    got = out[0::2] + 1j * out[1::2]
    ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
    assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("nz", [16, 32, 64, 128, 256, 512, 1024])
def test_fourxz_lines(nz):
    """r2c keeps modes 0..nz2 scaled by 1/nz; c2r zeroes modes > nz2, is
    unscaled, and ignores Im X[0]."""
    L = pyoracle.lib()
    nz1 = 2 * (nz // 3)
    nz2 = nz1 // 2 - 1
    h = L.orc_fft_create(nz // 2)
    work = np.zeros(2 * (3 * (nz // 2) + 1))
    rng = np.random.default_rng(nz)
    phys = rng.standard_normal(nz)
    fou = np.zeros(2 * (nz2 + 1))
    L.orc_r2c_line(h, nz, nz2, D(phys), D(fou), D(work))
    ref = np.fft.rfft(phys)[:nz2 + 1] / nz
    got = fou[0::2] + 1j * fou[1::2]
    assert np.abs(got - ref).max() <= 1e-15 * max(1.0, np.abs(ref).max()) * 8
    X = rng.standard_normal(nz2 + 1) + 1j * rng.standard_normal(nz2 + 1)
    fin = np.ascontiguousarray(np.stack([X.real, X.imag], -1).ravel())
    out = np.zeros(nz)
    L.orc_c2r_line(h, nz, nz2, D(fin), D(out), D(work))
    full = np.zeros(nz // 2 + 1, dtype=complex)
    full[:nz2 + 1] = X
    full[0] = X[0].real
    ref = np.fft.irfft(full, nz) * nz
    assert np.abs(out - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
    L.orc_fft_destroy(h)


@pytest.mark.parametrize("n", [8, 32, 96, 128, 256, 384, 512, 1024])
def test_cosftx_lines(n):
    """REDFT10 x 1/n (iopt < 0) and REDFT01 x 0.5 (iopt >= 0); scipy's
    type-2/type-3 DCTs with norm=None are the same definitions."""
    L = pyoracle.lib()
    h = L.orc_fft_create(n)
    work = np.zeros(4 * n)
    rng = np.random.default_rng(n + 1)
    x = rng.standard_normal(n)
    c = x.copy()
    L.orc_dct_line(h, n, D(c), -1, D(work))
    ref = sfft.dct(x, type=2) / n
    assert np.abs(c - ref).max() <= 1e-14 * max(1.0, np.abs(ref).max())
    c = x.copy()
    L.orc_dct_line(h, n, D(c), 1, D(work))
    ref = sfft.dct(x, type=3) * 0.5
    assert np.abs(c - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
    # forward then inverse: REDFT01(REDFT10(x))/(2n) = x, so (x/n)*0.5*2 = x
    c = x.copy()
    L.orc_dct_line(h, n, D(c), -1, D(work))
    L.orc_dct_line(h, n, D(c), 1, D(work))
    assert np.abs(c - x).max() <= 1e-13
    L.orc_fft_destroy(h)
