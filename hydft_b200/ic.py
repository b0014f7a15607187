"""Seeded initial conditions that both the CUDA path and any checker can
reproduce bit for bit.

HyDFT's `random` initial condition (src/model/initial.f90:47-58) draws from
gfortran's intrinsic generator, which cannot be reproduced outside gfortran.
This module replaces it with a counter-based stream: value q of stream `seed`
is splitmix64's output for state seed*2^32 + q, i.e.

    z = (seed << 32) + (q + 1) * 0x9E3779B97F4A7C15   (mod 2^64)
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9
    z = (z ^ (z >> 27)) * 0x94D049BB133111EB
    z =  z ^ (z >> 31)
    u = (z >> 11) * 2^-53                               in [0, 1)

Fields use the reference's Fortran layout: shape (nz, ny, nx), C order.
"""
import numpy as np

_M64 = (1 << 64) - 1


def splitmix_uniform(seed, count, offset=0):
    """`count` uniforms in [0,1) from counters offset..offset+count-1."""
    with np.errstate(over="ignore"):
        q = np.arange(offset, offset + count, dtype=np.uint64)
        z = (np.uint64((int(seed) << 32) & _M64) + (q + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _mask(nx, ny, nz, lx, ly, lz):
    """2/3-rule mask on the r2c half spectrum, as grid_init builds it
    (src/core/grid.f90:89-112)."""
    twopi = 2.0 * np.pi
    kx = twopi * np.arange(nx // 2 + 1) / lx
    ky = twopi * np.where(np.arange(ny) <= ny // 2, np.arange(ny), np.arange(ny) - ny) / ly if ny > 1 else np.zeros(1)
    kz = twopi * np.where(np.arange(nz) <= nz // 2, np.arange(nz), np.arange(nz) - nz) / lz if nz > 1 else np.zeros(1)
    kxc = twopi * (nx // 2) / lx * (2.0 / 3.0)
    kyc = twopi * (ny // 2) / ly * (2.0 / 3.0) if ny > 1 else np.inf
    kzc = twopi * (nz // 2) / lz * (2.0 / 3.0) if nz > 1 else np.inf
    KZ, KY, KX = np.meshgrid(kz, ky, kx, indexing="ij")
    keep = (np.abs(KX) < kxc) & (np.abs(KY) < kyc) & (np.abs(KZ) < kzc)
    return keep.astype(np.float64), KX, KY, KZ


def random_field(nx, ny, nz, lx, ly, lz, seed):
    """Zero-mean, unit-rms, 2/3-dealiased random field: the reference's
    `random` recipe (initial.f90:47-58: uniform - 1/2, dealias, remove the
    mean, normalise the rms) on the counter-based stream above."""
    d = splitmix_uniform(seed, nx * ny * nz).reshape(nz, ny, nx) - 0.5
    mask, _, _, _ = _mask(nx, ny, nz, lx, ly, lz)
    d = np.fft.irfftn(np.fft.rfftn(d) * mask, s=(nz, ny, nx), axes=(0, 1, 2))
    d -= d.mean()
    rms = np.sqrt(np.mean(d * d))
    return d / rms if rms > 0 else d


def gaussian_spectrum_field(nx, ny, nz, lx, ly, lz, seed, qc=1.0):
    """Zero-mean, unit-rms Gaussian random field whose power spectrum is
    proportional to exp(-(q/qc)^2), 2/3-dealiased.  White Gaussian noise
    (Box-Muller on the counter-based stream) is shaped in Fourier space by
    the amplitude exp(-(q/qc)^2/2)."""
    n = nx * ny * nz
    u1 = splitmix_uniform(seed, n, 0)
    u2 = splitmix_uniform(seed, n, n)
    g = np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)
    g = g.reshape(nz, ny, nx)
    mask, KX, KY, KZ = _mask(nx, ny, nz, lx, ly, lz)
    q2 = KX ** 2 + KY ** 2 + KZ ** 2
    amp = np.exp(-0.5 * q2 / (qc * qc)) * mask
    amp[0, 0, 0] = 0.0
    d = np.fft.irfftn(np.fft.rfftn(g) * amp, s=(nz, ny, nx), axes=(0, 1, 2))
    d -= d.mean()
    rms = np.sqrt(np.mean(d * d))
    return d / rms if rms > 0 else d


def mode_field(nx, ny, nz, lx, ly, lz, mode):
    """cos(k.r) of set_initial_condition's `mode` (initial.f90:36-46)."""
    twopi = 2.0 * np.pi
    kv = [twopi * mode[0] / lx, twopi * mode[1] / ly, twopi * mode[2] / lz]
    if ny == 1:
        kv[1] = 0.0
    if nz == 1:
        kv[2] = 0.0
    x = np.arange(nx) * (lx / nx)
    y = np.arange(ny) * (ly / ny)
    z = np.arange(nz) * (lz / nz)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return np.cos(kv[0] * X + kv[1] * Y + kv[2] * Z)
