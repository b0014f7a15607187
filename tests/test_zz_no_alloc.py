"""The allocation-free Fourier-Bessel transform, checked against the
allocating entry point.

hydft_gpu_fourier_bessel_noalloc is for callers that cannot allocate device
memory where they need the transform; it keeps its tables in a fixed scratch
array inside the library and works on device arrays the caller owns.  This
file is collected last so that a run stopping at the first failure has run
every other test; it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    import hydft_b200
    L = hydft_b200.lib()
    L.hydft_gpu_fourier_bessel_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                                   C.c_int, C.c_void_p]
    L.hydft_gpu_fourier_bessel_noalloc.restype = C.c_int
    L.hydft_gpu_create_error.restype = C.c_char_p
    return L


def _allocating(f, rmax, direction):
    from hydft_b200 import model
    return model.fourier_bessel(f, rmax, direction)


def _noalloc(L, torch, f, rmax, direction):
    dev_in = torch.tensor(f, dtype=torch.float64, device="cuda")
    dev_out = torch.full_like(dev_in, float("nan"))
    stream = torch.cuda.current_stream()
    rc = L.hydft_gpu_fourier_bessel_noalloc(dev_in.data_ptr(), dev_out.data_ptr(), f.size, rmax,
                                            direction, stream.cuda_stream)
    assert rc == 0, L.hydft_gpu_create_error()
    stream.synchronize()
    return dev_out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    L = _lib()
    # two calls in a row with different sizes and directions: each call must
    # rebuild the scratch tables it needs, whatever the previous call left
    nr1, rmax1 = 4096, 60.0
    r1 = rmax1 / (nr1 + 1) * np.arange(1, nr1 + 1)
    f1 = np.exp(-r1) * (1.0 + 0.3 * np.cos(r1))
    nr2, rmax2 = 3000, 45.0
    k2 = np.pi / (rmax2) * np.arange(1, nr2 + 1)
    f2 = 8.0 * np.pi / (k2 ** 2 + 1.0) ** 2
    for f, rmax, direction in ((f1, rmax1, 0), (f2, rmax2, 1)):
        ref = _allocating(f, rmax, direction)
        got = _noalloc(L, torch, f, rmax, direction)
        assert np.all(np.isfinite(got))
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_noalloc_at_the_maximum_size_then_a_smaller_one():
    import torch
    L = _lib()
    # n = 8192 fills the scratch array exactly and needs the largest shared
    # sine table; the smaller call after it must not see the larger call's
    # leftover tables
    nmax = 8192
    rmax = 80.0
    r = rmax / (nmax + 1) * np.arange(1, nmax + 1)
    fa = np.exp(-0.5 * r) * np.sin(0.7 * r) / (1.0 + r)
    nb, rmaxb = 1024, 30.0
    kb = np.pi / rmaxb * np.arange(1, nb + 1)
    fb = np.exp(-0.1 * kb * kb)
    for f, rm, direction in ((fa, rmax, 0), (fb, rmaxb, 1), (fa, rmax, 1)):
        ref = _allocating(f, rm, direction)
        got = _noalloc(L, torch, f, rm, direction)
        assert np.all(np.isfinite(got))
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_noalloc_rejects_overlapping_arrays():
    import torch
    L = _lib()
    n = 256
    dev = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    for off in (0, 1, n - 1):
        rc = L.hydft_gpu_fourier_bessel_noalloc(dev.data_ptr(), dev.data_ptr() + 8 * off, n, 60.0, 0, None)
        assert rc == 1
        assert b"overlap" in L.hydft_gpu_create_error()
    # adjacent, not overlapping: accepted
    rc = L.hydft_gpu_fourier_bessel_noalloc(dev.data_ptr(), dev.data_ptr() + 8 * n, n, 60.0, 0, None)
    assert rc == 0, L.hydft_gpu_create_error()
    torch.cuda.synchronize()


def test_noalloc_rejects_sizes_beyond_the_scratch():
    import torch
    L = _lib()
    n = 8193
    dev = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc = L.hydft_gpu_fourier_bessel_noalloc(dev.data_ptr(), dev.data_ptr(), n, 60.0, 0, None)
    assert rc == 1
    assert b"8192" in L.hydft_gpu_create_error()
