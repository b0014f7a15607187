"""The reference's integration tests (test/test_conservation.f90,
test_mode_newtonian.f90, test_mode_maxwell.f90, test_driven_mode.f90,
test_ground_state.f90) run on the GPU path through the C ABI, with the
reference's thresholds.  Linear theory (dispersion, chi, K(k)) comes from the
oracle, which restates the reference's linear-response code; the fits are
the oracle's restatements of python/hydft_io.py's.
"""
import numpy as np
import pytest

from hydft_b200 import ic

pytestmark = pytest.mark.gpu

TWOPI = 2.0 * np.pi
HNC = dict(hnc_nr=4096, hnc_rmax=60.0)


@pytest.fixture(scope="module")
def hg():
    import hydft_b200
    hydft_b200.lib()
    return hydft_b200


def pair(hg, orc, **kw):
    m = hg.Model(hg.default_params(**kw))
    k, c = m.structure()
    st = orc.Structure(k, c, m.scalar("n0"), m.scalar("u_ex"), m.scalar("du_dgamma"), True)
    okw = {kk: v for kk, v in kw.items() if kk != "gpu_precision"}
    return m, orc.Model(orc.params(**okw), st)


@pytest.mark.parametrize("closure,eta,tau,prec", [("newtonian", 2.0, 0.0, "fp64"), ("maxwell", 0.2, 2.0, "fp64"),
                                                  ("newtonian", 2.0, 0.0, "fp32")])
def test_conservation(hg, closure, eta, tau, prec):
    m = hg.Model(hg.default_params(kind="ion", gamma=2.0, kappa=0.1, nx=32, ny=4, nz=1, lx=20.0, ly=5.0,
                                   transport="constant", eta=eta, closure=closure, tau_model="constant",
                                   tau=tau, cfl=0.3, gpu_precision=prec, **HNC))
    d = ic.random_field(32, 4, 1, 20.0, 5.0, 1.0, seed=7)
    m.set_state(m.scalar("n0") * (1 + 0.02 * d))
    mass0, mom0, ek0, fe0, _, _ = m.budgets()
    for _ in range(100):
        m.compute_dt()
        m.advance(1)
    mass, mom, ek, fe, _, _ = m.budgets()
    tol = 1e-12 if prec == "fp64" else 1e-6
    assert abs(mass / mass0 - 1) < tol
    assert np.abs(mom - mom0).max() / (mass0 * np.sqrt(ek / mass0)) < (1e-12 if prec == "fp64" else 1e-5)
    assert ek > 0
    if closure == "newtonian":
        assert (ek + fe - ek0 - fe0) / abs(ek0 + fe0) < (1e-8 if prec == "fp64" else 1e-5)


def mode_run(hg, orc, kw, mode, tend, tfit):
    m, o = pair(hg, orc, **kw)
    m.set_initial_condition("mode", 1e-4, (mode, 0, 0))
    q = TWOPI * mode / kw["lx"]
    w = o.dispersion(q)
    ts, ys = [], []
    while m.t < tend:
        m.compute_dt()
        m.advance(1)
        ts.append(m.t)
        ys.append(m.mode(0, mode, 0, 0).real)
    om, ga, _ = orc.fit_damped_mode(np.array(ts), np.array(ys), tfit)
    m.close()
    return w, om, ga


@pytest.mark.parametrize("kind,prec", [("ion", "fp64"), ("electron", "fp64"), ("ion", "fp32")])
def test_mode_newtonian(hg, orc, kind, prec):
    kw = dict(kind=kind, gamma=1.0 if kind == "electron" else 2.0, kappa=0.1, rs=1.86, nx=32, ny=1, nz=1,
              lx=20.0, transport="constant", eta=0.1, closure="newtonian", cfl=0.1, gpu_precision=prec, **HNC)
    w, om, ga = mode_run(hg, orc, kw, 2, 100.0, 5.0)
    assert abs(om / w.real - 1) < 0.01
    assert abs(ga / w.imag - 1) < 0.03


def test_mode_maxwell(hg, orc):
    res = {}
    for closure, tau in (("newtonian", 0.0), ("maxwell", 3.0), ("maxwell", 0.02)):
        kw = dict(kind="ion", gamma=2.0, kappa=0.1, nx=32, ny=1, nz=1, lx=20.0, transport="constant", eta=0.1,
                  closure=closure, tau_model="constant", tau=tau, cfl=0.1, **HNC)
        w, om, ga = mode_run(hg, orc, kw, 2, 120.0, 20.0)
        assert abs(om / w.real - 1) < 0.01
        assert abs(ga / w.imag - 1) < 0.05
        res[tau] = (om, ga)
    om_n, ga_n = res[0.0]
    om_s, ga_s = res[0.02]
    assert abs(om_s / om_n - 1) < 0.01 and abs(ga_s / ga_n - 1) < 0.05


@pytest.mark.parametrize("closure,tau", [("newtonian", 0.0), ("maxwell", 1.0)])
def test_driven_mode(hg, orc, closure, tau):
    mode, amp = 2, 1e-5
    kw = dict(kind="ion", gamma=2.0, kappa=0.1, nx=32, ny=1, nz=1, lx=20.0, transport="constant", eta=0.3,
              closure=closure, tau_model="constant", tau=tau, cfl=0.1, vext="driven", vext_amplitude=amp,
              vext_mode=(mode, 0, 0), vext_ramp=10.0, **HNC)
    m, o = pair(hg, orc, **kw)
    q = TWOPI * mode / kw["lx"]
    wd = 0.7 * q * np.sqrt(o.c2(q))
    m.set_scalar("ext_omega", wd)
    ts, zs = [], []
    while m.t < 300.0:
        m.compute_dt()
        m.advance(1)
        ts.append(m.t)
        zs.append(m.mode(0, mode, 0, 0))
    a, scatter = orc.fit_driven_response(np.array(ts), np.array(zs), wd, 250.0)
    chi_sim = 2.0 * a / amp
    chi_lin = o.chi(q, wd)
    assert abs(chi_sim - chi_lin) / abs(chi_lin) < 0.02
    assert scatter < 0.05
    m.close()


@pytest.mark.parametrize("kind", ["ion", "electron"])
def test_ground_state(hg, orc, kind):
    mode, amp = 1, 1e-3
    kw = dict(kind=kind, gamma=1.0 if kind == "electron" else 2.0, kappa=0.1, rs=1.86, nx=32, ny=1, nz=1,
              lx=20.0, transport="constant", eta=1.0, closure="newtonian", cfl=0.2, vext="mode",
              vext_amplitude=amp, vext_mode=(mode, 0, 0), **HNC)
    m, o = pair(hg, orc, **kw)
    while m.t < 150.0:
        m.compute_dt()
        m.advance(1)
    n = m.get_state()[0]
    # mu[n] + v_ext is uniform in the ground state (evaluated by the oracle's functional)
    mu = o.mu_total(n, o.fwd(n))
    x = np.arange(32) * 20.0 / 32
    v = amp * np.cos(TWOPI * mode * x / 20.0)
    tot = mu.ravel() + v
    spread = (tot.max() - tot.min()) / amp
    q = TWOPI * mode / kw["lx"]
    dnk = m.mode(0, mode, 0, 0)
    pred = -0.5 * amp / o.kernel(q)
    assert spread < 2e-3
    assert abs(dnk - pred) / abs(pred) < 1e-2
    m.close()
