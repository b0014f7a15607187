"""Ensembles (hydft_batch_*): many models advanced by one graph launch per
step give the same fields as each model advanced alone.

The members differ in grid, species, Gamma, kappa and closure; every member
is stepped at its own dt.  The kernels are deterministic, so a member of the
ensemble and the same model on its own agree to the last bit.
"""
import numpy as np
import pytest

from hydft_b200 import ic

pytestmark = pytest.mark.gpu

HNC = dict(hnc_nr=2048, hnc_rmax=40.0)
MEMBERS = [
    dict(kind="ion", gamma=10.0, kappa=1.0, transport="yukawa_fit", nx=16, ny=16, nz=16,
         lx=10.0, ly=10.0, lz=10.0, **HNC),
    dict(kind="ion", gamma=30.0, kappa=2.0, closure="maxwell", transport="yukawa_fit", tau_model="ichimaru",
         nx=32, ny=16, nz=8, lx=16.0, ly=8.0, lz=4.0, **HNC),
    dict(kind="electron", rs=1.0, theta=1.0, transport="constant", eta=0.2, nx=16, ny=8, nz=8,
         lx=12.0, ly=6.0, lz=6.0, vext="driven", vext_amplitude=1e-3, vext_mode=(1, 0, 0), vext_omega=1.0, **HNC),
    dict(kind="ion", gamma=10.0, kappa=1.0, transport="yukawa_fit", nx=16, ny=16, nz=16,
         lx=10.0, ly=10.0, lz=10.0, gpu_precision="fp32", **HNC),
    # grids with register FFT plans on every axis: members of equal shape
    # step as one group (shared launches, per-member argument tables)
    dict(kind="ion", gamma=5.0, kappa=0.5, transport="yukawa_fit", nx=32, ny=32, nz=32,
         lx=20.0, ly=20.0, lz=20.0, gpu_precision="fp32", **HNC),
    dict(kind="ion", gamma=40.0, kappa=2.5, transport="yukawa_fit", nx=32, ny=32, nz=32,
         lx=20.0, ly=20.0, lz=20.0, gpu_precision="fp32", **HNC),
    dict(kind="ion", gamma=20.0, kappa=1.5, closure="maxwell", transport="yukawa_fit", tau_model="ichimaru",
         nx=48, ny=32, nz=32, lx=30.0, ly=20.0, lz=20.0, gpu_precision="fp32", **HNC),
    dict(kind="ion", gamma=3.0, kappa=0.8, closure="maxwell", transport="yukawa_fit", tau_model="ichimaru",
         nx=48, ny=32, nz=32, lx=24.0, ly=16.0, lz=16.0, gpu_precision="fp32", **HNC),
    dict(kind="ion", gamma=8.0, kappa=1.0, transport="yukawa_fit", nx=32, ny=48, nz=64,
         lx=16.0, ly=24.0, lz=32.0, **HNC),
    dict(kind="electron", rs=1.0, theta=1.0, transport="constant", eta=0.2, nx=32, ny=32, nz=32,
         lx=12.0, ly=12.0, lz=12.0, vext="driven", vext_amplitude=1e-3, vext_mode=(1, 0, 0), vext_omega=1.0,
         gpu_precision="fp32", **HNC),
    dict(kind="electron", rs=2.0, theta=0.5, transport="constant", eta=0.1, nx=32, ny=32, nz=32,
         lx=12.0, ly=12.0, lz=12.0, vext="driven", vext_amplitude=1e-3, vext_mode=(1, 0, 0), vext_omega=0.7,
         gpu_precision="fp32", **HNC),
]


@pytest.fixture(scope="module")
def hg():
    import hydft_b200
    hydft_b200.lib()
    return hydft_b200


def init(m, i):
    p = m.p
    n0 = m.scalar("n0")
    n = n0 * (1 + 0.01 * ic.random_field(m.nx, m.ny, m.nz, p.lx, p.ly, p.lz, 40 + i))
    mom = np.zeros((3,) + m.shape)
    mom[0] = 0.005 * n0 * ic.random_field(m.nx, m.ny, m.nz, p.lx, p.ly, p.lz, 50 + i)
    m.set_state(n, mom)
    m.compute_dt()


def test_batch_matches_members_alone(hg):
    params = [hg.default_params(**kw) for kw in MEMBERS]
    b = hg.Batch(params)
    try:
        assert len(b) == len(MEMBERS)
        for i, m in enumerate(b.members):
            init(m, i)
        b.advance(3)
        b.advance(2)
        # the 32^3 ion pair, the 48x32x32 Maxwell pair, the 32x48x64 member
        # and the electron pair step in groups; the 16-point grids alone
        groups, grouped = b.grouped()
        assert groups >= 4 and grouped >= 7, (groups, grouped)
        for i, kw in enumerate(MEMBERS):
            alone = hg.Model(hg.default_params(**kw))
            init(alone, i)
            alone.advance(5)
            got, ref = b.members[i].get_state(), alone.get_state()
            for x, y in zip(got, ref):
                if y is not None:
                    assert np.array_equal(x, y), "member %d differs from the model alone" % i
            assert b.members[i].step == alone.step == 5
            assert abs(b.members[i].t - alone.t) == 0.0
            alone.close()
        # the member handles stay usable between ensemble steps
        mass0 = b.members[1].budgets()[0]
        b.advance(1)
        assert abs(b.members[1].budgets()[0] - mass0) < 1e-12 * abs(mass0)
        assert b.launch_count() > 0
    finally:
        b.close()


def test_batch_reports_the_failing_member(hg):
    params = [hg.default_params(**MEMBERS[0]), hg.default_params(**MEMBERS[0])]
    b = hg.Batch(params)
    try:
        init(b.members[0], 0)
        # member 1 has no dt
        with pytest.raises(hg.HydftError):
            b.advance(1)
        assert b.failed_member() == 1
    finally:
        b.close()
