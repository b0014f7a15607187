"""The benchmark configurations as parity cases (the 256^3 Maxwell step is
bench.py's workload).

C1 (32^3 Yukawa ions, Newtonian, FP64, single mode 1e-3, dt 0.01): the GPU
path against the oracle after 40 steps, 1e-10 relative per field.
C3 (128^3 electrons, Thomas-Fermi + gradient + Hartree + RY, driven at
q = 2 pi/L (3,0,0)): FP32 against FP64 on the GPU after 40 steps, within
the 1e-5 relative field error of the FP32 path.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TWOPI = 2.0 * np.pi


@pytest.fixture(scope="module")
def hg():
    import hydft_b200
    hydft_b200.lib()
    return hydft_b200


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_c1_ion_newtonian_32_matches_oracle(hg, orc):
    kw = dict(kind="ion", gamma=10.0, kappa=1.0, nx=32, ny=32, nz=32, lx=20.0, ly=20.0, lz=20.0,
              closure="newtonian", transport="yukawa_fit", hnc_nr=4096, hnc_rmax=80.0, dt=0.01)
    m = hg.Model(hg.default_params(**kw))
    k, c = m.structure()
    st = orc.Structure(k, c, m.scalar("n0"), m.scalar("u_ex"), m.scalar("du_dgamma"), True)
    o = orc.Model(orc.params(**kw), st)
    n0 = m.scalar("n0")
    x = np.arange(32) * 20.0 / 32
    n = np.broadcast_to(n0 * (1 + 1e-3 * np.cos(TWOPI * x / 20.0)), (32, 32, 32)).copy()
    m.set_state(n)
    o.set_state(n)
    m.advance(40)
    o.advance(40)
    g, r = m.get_state(), (o.n, o.mom)
    assert rel(g[0] - n0, r[0] - n0) < 1e-10
    assert rel(g[1], r[1]) < 1e-10
    m.close()


def test_c3_electron_driven_128_fp32_vs_fp64(hg):
    base = dict(kind="electron", rs=1.0, theta=1.0, nx=128, ny=128, nz=128, lx=40.0, ly=40.0, lz=40.0,
                closure="newtonian", transport="constant", eta=0.2, vext="driven", vext_amplitude=1e-4,
                vext_mode=(3, 0, 0), vext_omega=1.0, hnc_nr=4096, hnc_rmax=80.0)
    m64 = hg.Model(hg.default_params(gpu_precision="fp64", **base))
    dt = m64.compute_dt()
    k, c = m64.structure()
    st = dict(k=k, c=c, u_ex=m64.scalar("u_ex"), du_dgamma=m64.scalar("du_dgamma"))
    m32 = hg.Model(hg.default_params(gpu_precision="fp32", **base), structure=st)
    m32.set_time(0.0, dt)
    m64.advance(40)
    m32.advance(40)
    a, b = m32.get_state(), m64.get_state()
    n0 = m64.scalar("n0")
    assert rel(a[0] - n0, b[0] - n0) < 1e-5
    assert rel(a[1], b[1]) < 1e-5
    # the drive has put momentum into the driven mode
    assert abs(m64.mode(1, 3, 0, 0)) > 0
    m32.close()
    m64.close()
