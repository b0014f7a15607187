"""The reference's own known-answer tests, restated against the CPU oracle
with the reference's thresholds.  These pin the oracle before it is trusted
as the reference for the CUDA path.

  test/test_fft.f90:21-52        FFT round trip and normalised amplitudes
  test/test_ops.f90:30-71        derivatives, Laplacian, div, convolution, dealias
  test/test_fermi_dirac.f90:15-52  Fermi-Dirac limits, I_1/2(0), inverse
  test/test_hnc.f90:25-35        Fourier-Bessel transform of exp(-r)
"""
import numpy as np
import pytest

TWOPI = 2.0 * np.pi


def _spec(orc, nx, ny, nz, lx, ly, lz):
    p = orc.params(nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, lz=lz, terms="ideal")
    return orc.Model(p)


def test_fft_1d(orc):
    # test_fft.f90:21-36
    m = _spec(orc, 64, 1, 1, TWOPI, TWOPI, TWOPI)
    x = np.arange(64) * TWOPI / 64
    u = (1.5 + 0.3 * np.cos(3 * x) + 0.2 * np.sin(5 * x)).reshape(1, 1, 64)
    F = orc.FFT3(64, 1, 1)
    uh = F.fwd(u)
    v = F.bwd(uh)
    assert np.abs(u - v).max() < 1e-13
    assert abs(uh[0, 0, 0] - 1.5) < 1e-13
    assert abs(uh[0, 0, 3] - 0.15) < 1e-13
    assert abs(uh[0, 0, 5] + 0.1j) < 1e-13
    assert abs(m.mode(u, 3, 0, 0) - 0.15) < 1e-13


def test_fft_3d(orc):
    # test_fft.f90:38-52
    nx, ny, nz = 16, 12, 8
    m = _spec(orc, nx, ny, nz, TWOPI, 4.0, 1.0)
    x = np.arange(nx) * TWOPI / nx
    y = np.arange(ny) * 4.0 / ny
    z = np.arange(nz) * 1.0 / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    u = 0.7 + np.cos(2 * X) * np.sin(TWOPI * Y / 4.0) + 0.4 * np.cos(TWOPI * 2.0 * Z)
    F = orc.FFT3(nx, ny, nz)
    v = F.bwd(F.fwd(u))
    assert np.abs(u - v).max() < 1e-13
    assert abs(m.mode(u, 0, 0, 2) - 0.2) < 1e-13
    assert abs(m.mode(u, 2, 1, 0) + 0.25j) < 1e-13


def test_fft_matches_numpy(orc):
    # the FFTW r2c/c2r conventions of src/core/fft.f90:51-69
    rng = np.random.default_rng(3)
    for (nx, ny, nz) in [(32, 32, 32), (48, 24, 12), (96, 1, 1), (20, 6, 1)]:
        u = rng.standard_normal((nz, ny, nx))
        F = orc.FFT3(nx, ny, nz)
        uh = F.fwd(u)
        ref = np.fft.rfftn(u) / u.size
        assert np.abs(uh - ref).max() < 1e-14 * max(1.0, np.abs(ref).max())
        assert np.abs(F.bwd(uh) - u).max() < 1e-13


def test_ops(orc):
    # test_ops.f90:30-71 on a 32x16x1 grid
    import ctypes as C
    nx, ny, nz = 32, 16, 1
    lx, ly = TWOPI, 4.0
    m = _spec(orc, nx, ny, nz, lx, ly, 1.0)
    L = orc.lib()
    spc = L.orc_model_spec(m.h)
    x = np.arange(nx) * lx / nx
    y = np.arange(ny) * ly / ny
    Y, X = np.meshgrid(y, x, indexing="ij")
    u = (np.sin(2 * X) * np.cos(TWOPI * Y / ly)).reshape(1, ny, nx).copy()
    du = np.zeros((3, 1, ny, nx))
    L.orc_spec_grad.argtypes = [C.c_void_p] * 3
    L.orc_spec_grad(spc, orc._ptr(u), orc._ptr(du))
    ex = 2 * np.cos(2 * X) * np.cos(TWOPI * Y / ly)
    assert np.abs(du[0, 0] - ex).max() < 1e-12
    ex = -(TWOPI / ly) * np.sin(2 * X) * np.sin(TWOPI * Y / ly)
    assert np.abs(du[1, 0] - ex).max() < 1e-12
    assert np.abs(du[2]).max() < 1e-14
    lu = np.zeros((1, ny, nx))
    L.orc_spec_lap.argtypes = [C.c_void_p] * 3
    L.orc_spec_lap(spc, orc._ptr(u), orc._ptr(lu))
    ex = -(4.0 + (TWOPI / ly) ** 2) * u
    assert np.abs(lu - ex).max() < 1e-11
    v = np.zeros((3, 1, ny, nx))
    v[0] = du[0]
    v[1] = du[1]
    dv = np.zeros((1, ny, nx))
    L.orc_spec_div.argtypes = [C.c_void_p] * 3
    L.orc_spec_div(spc, orc._ptr(v), orc._ptr(dv))
    assert np.abs(dv - ex).max() < 1e-11
    # convolution with 1/(1+k^2)
    kx = TWOPI * np.arange(nx // 2 + 1) / lx
    ky = TWOPI * np.fft.fftfreq(ny, 1.0 / ny) / ly
    KY, KX = np.meshgrid(ky, kx, indexing="ij")
    kern = (1.0 / (1.0 + KX ** 2 + KY ** 2)).reshape(1, ny, nx // 2 + 1).copy()
    uh = m.fwd(u)
    cu = np.zeros((1, ny, nx))
    L.orc_spec_convolve.argtypes = [C.c_void_p] * 4
    L.orc_spec_convolve(spc, orc._ptr(kern), orc._ptr(uh), orc._ptr(cu))
    ex = u / (1.0 + 4.0 + (TWOPI / ly) ** 2)
    assert np.abs(cu - ex).max() < 1e-13
    # dealias: cos(12x) goes, cos(10x) stays
    u2 = (np.cos(12 * X) + np.cos(10 * X)).reshape(1, ny, nx).copy()
    L.orc_spec_dealias.argtypes = [C.c_void_p] * 2
    L.orc_spec_dealias(spc, orc._ptr(u2))
    assert np.abs(u2[0] - np.cos(10 * X)).max() < 1e-13
    assert abs(m.get("kmax_dealiased") - np.sqrt(100.0 + (TWOPI * 5.0 / ly) ** 2)) < 1e-12
    L.orc_spec_mean.restype = C.c_double
    L.orc_spec_mean.argtypes = [C.c_void_p] * 2
    u3 = (3.0 + du[0]).copy()
    assert abs(L.orc_spec_mean(spc, orc._ptr(u3)) - 3.0) < 1e-13


def test_fermi_dirac(orc):
    # test_fermi_dirac.f90:15-52
    sp = np.sqrt(np.pi)
    a = -20.0
    assert abs(orc.fd("ip12", a) / (0.5 * sp * np.exp(a)) - 1) < 1e-8
    assert abs(orc.fd("im12", a) / (sp * np.exp(a)) - 1) < 1e-8
    assert abs(orc.fd("ip32", a) / (0.75 * sp * np.exp(a)) - 1) < 1e-8
    a = 250.0
    ex = (2.0 / 3.0) * a ** 1.5 * (1 + np.pi ** 2 / (8 * a * a))
    assert abs(orc.fd("ip12", a) / ex - 1) < 1e-8
    ex = 2 * np.sqrt(a) * (1 - np.pi ** 2 / (24 * a * a))
    assert abs(orc.fd("im12", a) / ex - 1) < 1e-8
    assert abs(orc.fd("ip12", 300 - 1e-9) / orc.fd("ip12", 300 + 1e-9) - 1) < 1e-8
    assert abs(orc.fd("ip12", -30 - 1e-9) / orc.fd("ip12", -30 + 1e-9) - 1) < 1e-8
    assert abs(orc.fd("ip12", 0.0) - 0.678093895) < 1e-8
    hh = 1e-4
    for ia in range(10):
        a = -5.0 + 4.7 * ia
        d = (orc.fd("ip12", a + hh) - orc.fd("ip12", a - hh)) / (2 * hh)
        assert abs(d / (0.5 * orc.fd("im12", a)) - 1) < 1e-7
        d = (orc.fd("ip32", a + hh) - orc.fd("ip32", a - hh)) / (2 * hh)
        assert abs(d / (1.5 * orc.fd("ip12", a)) - 1) < 1e-7
        d = (orc.fd("im12", a + hh) - orc.fd("im12", a - hh)) / (2 * hh)
        assert abs(d / orc.fd("dim12", a) - 1) < 1e-6
        d = (orc.fd("dim12", a + hh) - orc.fd("dim12", a - hh)) / (2 * hh)
        assert abs(d / orc.fd("d2im12", a) - 1) < 1e-5
        d = (orc.fd("xi", a + hh) - orc.fd("xi", a - hh)) / (2 * hh)
        assert abs(d / orc.fd("dxi", a) - 1) < 1e-5
    for ia in range(23):
        a = -25.0 + 13.3 * ia
        y = orc.fd("ip12", a)
        v, st = orc.fd_alpha_from_ip12(y)
        assert st == 0
        assert abs(v - a) < 1e-9 * max(1.0, abs(a))
    _, st = orc.fd_alpha_from_ip12(0.0)
    assert st == 1   # the reference's fatal for y <= 0 (fermi_dirac.f90:245)


def test_fourier_bessel(orc):
    # test_hnc.f90:25-35
    nr, rmax = 4096, 60.0
    dr = rmax / (nr + 1)
    r = dr * np.arange(1, nr + 1)
    k = np.pi / ((nr + 1) * dr) * np.arange(1, nr + 1)
    fr = np.exp(-r)
    fk = orc.fb_r2k(fr, rmax)
    sel = k < 20.0
    assert np.abs(fk[sel] * (k[sel] ** 2 + 1) ** 2 / (8 * np.pi) - 1).max() < 1e-4
    assert np.abs(orc.fb_k2r(fk, rmax) - fr).max() < 1e-12


def test_dst_matches_scipy(orc):
    import scipy.fft as sf
    rng = np.random.default_rng(1)
    for n in (7, 100, 4096):
        x = rng.standard_normal(n)
        y = orc.dst1(x)
        assert np.abs(y - sf.dst(x, type=1)).max() < 1e-12 * max(1.0, np.abs(y).max())
