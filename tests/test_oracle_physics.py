"""The reference's integration and consistency tests restated against the
CPU oracle, with the reference's thresholds:

  test/test_kernels.f90:19-70        K_i(k) vs finite difference of add_mu (2e-4)
  test/test_conservation.f90:33-53   mass/momentum 1e-12, Newtonian energy 1e-8
  test/test_mode_newtonian.f90:37-60 omega 1 %, gamma 3 %
  test/test_mode_maxwell.f90:20-64   omega 1 %, gamma 5 %, tau -> 0 limit
  test/test_driven_mode.f90:37-68    chi 2 %, scatter 5 %
  test/test_ground_state.f90:36-62   mu + v_ext spread 2e-3, dn_k 1 %
  test/test_hnc.f90:37-76            OCP/Yukawa/HM structure checks

The conservation test's `random` initial condition comes from the seeded
counter-based stream of hydft_b200.ic (the reference draws from gfortran's
intrinsic generator, which cannot be reproduced).
"""
import os

import numpy as np
import pytest

from hydft_b200 import ic

TWOPI = 2.0 * np.pi
N0 = 3.0 / (4.0 * np.pi)


@pytest.mark.parametrize("kind,terms", [("ion", "ideal,hartree,ry"),
                                        ("electron", "tf,gradient,hartree,ry"),
                                        ("electron", "tf,gradient,ry")])
def test_kernels(orc, kind, terms):
    p = orc.params(kind=kind, terms=terms, gamma=1.0 if kind == "electron" else 2.0,
                   kappa=0.1, rs=1.86, nx=64, ny=1, nz=1, lx=20.0, hnc_nr=4096,
                   hnc_rmax=60.0, transport="constant", closure="newtonian")
    m = orc.Model(p)
    eps = 1e-6
    n0a = np.full(m.shape, m.get("n0"))
    n0hat = m.fwd(n0a)
    x = np.arange(64) * 20.0 / 64
    for mm in range(1, 7):
        k = TWOPI * mm / 20.0
        n = (m.get("n0") * (1 + eps * np.cos(k * x))).reshape(m.shape)
        nhat = m.fwd(n)
        for it in range(m.nterms()):
            mu = np.zeros(m.shape)
            mu0 = np.zeros(m.shape)
            m.term_add_mu(it, n, nhat, mu)
            m.term_add_mu(it, n0a, n0hat, mu0)
            kfd = 2.0 * m.mode(mu - mu0, mm, 0, 0).real / (eps * m.get("n0"))
            kan = m.term_kernel(it, k)
            assert abs(kfd - kan) / max(abs(kan), 1e-3) < 2e-4, (m.term_name(it), mm)
        mu = m.mu_total(n, nhat)
        mu0 = m.mu_total(n0a, n0hat)
        kfd = 2.0 * m.mode(mu - mu0, mm, 0, 0).real / (eps * m.get("n0"))
        kan = m.kernel(k)
        assert abs(kfd - kan) / abs(kan) < 2e-4


@pytest.mark.parametrize("closure,eta,tau", [("newtonian", 2.0, 0.0), ("maxwell", 0.2, 2.0)])
def test_conservation(orc, closure, eta, tau):
    p = orc.params(kind="ion", gamma=2.0, kappa=0.1, nx=32, ny=4, nz=1, lx=20.0, ly=5.0,
                   hnc_nr=4096, hnc_rmax=60.0, transport="constant", eta=eta,
                   closure=closure, tau_model="constant", tau=tau, cfl=0.3)
    m = orc.Model(p)
    d = ic.random_field(32, 4, 1, 20.0, 5.0, 1.0, seed=7)
    m.set_state(m.get("n0") * (1 + 0.02 * d))
    mass0, mom0, ek0, fe0 = m.budgets()
    for _ in range(100):
        m.compute_dt()
        m.advance()
    mass, mom, ek, fe = m.budgets()
    assert abs(mass / mass0 - 1) < 1e-12
    assert np.abs(mom - mom0).max() / (mass0 * np.sqrt(ek / mass0)) < 1e-12
    assert ek > 0
    if closure == "newtonian":
        assert (ek + fe - ek0 - fe0) / abs(ek0 + fe0) < 1e-8


def _mode_run(orc, p, mode, tend, tfit):
    m = orc.Model(p)
    m.set_ic("mode", 1e-4, (mode, 0, 0))
    q = TWOPI * mode / p.lx
    w = m.dispersion(q)
    ts, ys = [], []
    while m.t < tend:
        m.compute_dt()
        m.advance()
        ts.append(m.t)
        ys.append(m.mode(m.n, mode, 0, 0).real)
    om, ga, nz = orc.fit_damped_mode(np.array(ts), np.array(ys), tfit)
    return w, om, ga


@pytest.mark.parametrize("kind", ["ion", "electron"])
def test_mode_newtonian(orc, kind):
    p = orc.params(kind=kind, gamma=1.0 if kind == "electron" else 2.0, kappa=0.1, rs=1.86,
                   nx=32, lx=20.0, hnc_nr=4096, hnc_rmax=60.0, transport="constant",
                   eta=0.1, closure="newtonian", cfl=0.1)
    w, om, ga = _mode_run(orc, p, 2, 100.0, 5.0)
    assert abs(om / w.real - 1) < 0.01
    assert abs(ga / w.imag - 1) < 0.03


def test_mode_maxwell(orc):
    res = {}
    for closure, tau in (("newtonian", 0.0), ("maxwell", 3.0), ("maxwell", 0.02)):
        p = orc.params(kind="ion", gamma=2.0, kappa=0.1, nx=32, lx=20.0, hnc_nr=4096,
                       hnc_rmax=60.0, transport="constant", eta=0.1, closure=closure,
                       tau_model="constant", tau=tau, cfl=0.1)
        w, om, ga = _mode_run(orc, p, 2, 120.0, 20.0)
        assert abs(om / w.real - 1) < 0.01
        assert abs(ga / w.imag - 1) < 0.05
        res[tau] = (om, ga)
    om_n, ga_n = res[0.0]
    om_s, ga_s = res[0.02]
    assert abs(om_s / om_n - 1) < 0.01 and abs(ga_s / ga_n - 1) < 0.05


@pytest.mark.parametrize("closure,tau", [("newtonian", 0.0), ("maxwell", 1.0)])
def test_driven_mode(orc, closure, tau):
    mode, amp = 2, 1e-5
    p = orc.params(kind="ion", gamma=2.0, kappa=0.1, nx=32, lx=20.0, hnc_nr=4096,
                   hnc_rmax=60.0, transport="constant", eta=0.3, closure=closure,
                   tau_model="constant", tau=tau, cfl=0.1, vext="driven",
                   vext_amplitude=amp, vext_mode=(mode, 0, 0), vext_ramp=10.0)
    m = orc.Model(p)
    q = TWOPI * mode / p.lx
    wd = 0.7 * q * np.sqrt(m.c2(q))
    m.set("ext_omega", wd)
    m.set_ic("uniform", 0.0)
    ts, zs = [], []
    while m.t < 300.0:
        m.compute_dt()
        m.advance()
        ts.append(m.t)
        zs.append(m.mode(m.n, mode, 0, 0))
    a, scatter = orc.fit_driven_response(np.array(ts), np.array(zs), wd, 250.0)
    chi_sim = 2.0 * a / amp
    chi_lin = m.chi(q, wd)
    assert abs(chi_sim - chi_lin) / abs(chi_lin) < 0.02
    assert scatter < 0.05


@pytest.mark.parametrize("kind", ["ion", "electron"])
def test_ground_state(orc, kind):
    mode, amp = 1, 1e-3
    p = orc.params(kind=kind, gamma=1.0 if kind == "electron" else 2.0, kappa=0.1, rs=1.86,
                   nx=32, lx=20.0, hnc_nr=4096, hnc_rmax=60.0, transport="constant",
                   eta=1.0, closure="newtonian", cfl=0.2, vext="mode",
                   vext_amplitude=amp, vext_mode=(mode, 0, 0))
    m = orc.Model(p)
    m.set_ic("uniform", 0.0)
    while m.t < 150.0:
        m.compute_dt()
        m.advance()
    n = m.n.copy()
    mu = m.mu_total(n, m.fwd(n))
    tot = mu + m.vext_v
    spread = (tot.max() - tot.min()) / amp
    q = TWOPI * mode / p.lx
    dnk = m.mode(n, mode, 0, 0)
    pred = -0.5 * amp / m.kernel(q)
    assert spread < 2e-3
    assert abs(dnk - pred) / abs(pred) < 1e-2


def test_hnc_ocp_and_hm(orc):
    # test_hnc.f90:37-76 (the Gamma = 50 OCP and the Yukawa(150, 0.1) cases
    # are in test_hnc_strong below)
    gam = 10.0
    res = orc.hnc_solve(orc.make_pot("coulomb", gam), N0, 8192, 80.0, 1e-9, 0.2, 5000)
    ufit = -0.897744 * gam + 0.95043 * gam ** 0.25 + 0.18956 * gam ** -0.25 - 0.81487
    assert res.converged
    assert abs(res.u_ex / ufit - 1) < 0.03
    assert abs(res.g[0]) < 1e-6 and abs(res.g[-1] - 1) < 1e-6
    assert abs(res.sk[0] / (res.k[0] ** 2 / (3 * gam)) - 1) < 0.05
    st = orc.structure_from_hnc(orc.make_pot("yukawa", 5.0, 1.0), N0, 8192, 80.0, 1e-9, 0.2,
                                5000, with_derivative=True)
    q = 0.5
    smf = (q * q + 1.0) / (q * q + 1.0 + 15.0)
    assert abs(st.s_of_k(q) / smf - 1) < 0.25
    assert st.u_ex < 0 and st.du_dgamma < 0
    res = orc.hnc_solve(orc.make_pot("hm", 1.0, 0.0, 2 * np.sqrt(np.pi / 1.86)), N0, 8192,
                        80.0, 1e-9, 0.2, 5000)
    assert res.converged
    assert 0 < res.g[0] < 1
    assert abs(res.sk[0] / (res.k[0] ** 2 / 3.0) - 1) < 0.05


@pytest.mark.skipif(not os.environ.get("HYDFT_SLOW"), reason="about 2 minutes; set HYDFT_SLOW=1")
def test_hnc_strong(orc):
    gam = 50.0
    res = orc.hnc_solve(orc.make_pot("coulomb", gam), N0, 8192, 80.0, 1e-9, 0.2, 5000)
    ufit = -0.897744 * gam + 0.95043 * gam ** 0.25 + 0.18956 * gam ** -0.25 - 0.81487
    assert res.converged and abs(res.u_ex / ufit - 1) < 0.03
    res = orc.hnc_solve(orc.make_pot("yukawa", 150.0, 0.1), N0, 8192, 80.0, 1e-8, 0.1, 20000)
    assert res.converged and res.g.max() > 1.5
