"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64: every result within 1e-10 relative (l2 over each field) of the oracle
on the same seeded inputs and the same structure table c(k).  FP32: within
1e-5.  The oracle restates the reference's FP64 FFTW path; see oracle/.
"""
import numpy as np
import pytest

from hydft_b200 import ic

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-5


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module")
def hg():
    import hydft_b200
    hydft_b200.lib()
    return hydft_b200


def pair(hg, orc, **kw):
    """A GPU model and an oracle model on the GPU's structure table."""
    m = hg.Model(hg.default_params(**kw))
    k, c = m.structure()
    st = None
    if k.size:
        st = orc.Structure(k, c, m.scalar("n0"), m.scalar("u_ex"), m.scalar("du_dgamma"), True)
    okw = {kk: v for kk, v in kw.items() if kk != "gpu_precision"}
    return m, orc.Model(orc.params(**okw), st)


def seeded_state(m, amp=0.02, seed=5, with_mom=True, with_pi=True):
    nx, ny, nz = m.nx, m.ny, m.nz
    p = m.p
    n0 = m.scalar("n0")
    n = n0 * (1 + amp * ic.random_field(nx, ny, nz, p.lx, p.ly, p.lz, seed))
    mom = np.zeros((3, nz, ny, nx))
    if with_mom:
        for d in range(m.scalar("ndim").__int__()):
            mom[d] = 0.01 * n0 * ic.random_field(nx, ny, nz, p.lx, p.ly, p.lz, seed + 10 + d)
    pi = None
    if m.has_pi and with_pi:
        pi = np.zeros((6, nz, ny, nx))
        for c in range(6):
            pi[c] = 1e-3 * ic.random_field(nx, ny, nz, p.lx, p.ly, p.lz, seed + 20 + c)
        if m.scalar("ndim") < 3:
            pass
    return n, mom, pi


ION = dict(kind="ion", gamma=10.0, kappa=1.0, hnc_nr=2048, hnc_rmax=40.0, transport="yukawa_fit")
ELEC = dict(kind="electron", rs=1.0, theta=1.0, hnc_nr=2048, hnc_rmax=40.0, transport="constant",
            eta=0.2)


def test_fd_table_and_inverse(hg, orc):
    t = hg.fd_table()
    to = orc.fd_table()
    assert t.shape == to.shape == (6601, 6)
    assert np.abs(t - to).max() / np.abs(to).max() < 1e-13
    a = np.linspace(-35.0, 320.0, 97)
    y = np.array([orc.fd("ip12", v) for v in a])
    al = hg.fd_alpha(y)
    ao = np.array([orc.fd_alpha_from_ip12(v)[0] for v in y])
    assert np.abs(al - ao).max() < 1e-9 * max(1.0, np.abs(ao).max())


def test_fourier_bessel_matches_oracle(hg, orc):
    from hydft_b200 import model
    nr, rmax = 4096, 60.0
    dr = rmax / (nr + 1)
    r = dr * np.arange(1, nr + 1)
    k = np.pi / ((nr + 1) * dr) * np.arange(1, nr + 1)
    fr = np.exp(-r)
    fk = model.fourier_bessel(fr, rmax, 0)
    assert np.abs(fk - orc.fb_r2k(fr, rmax)).max() < 1e-12 * np.abs(fk).max()
    # test_hnc.f90:25-35: transform of exp(-r) and the round trip
    sel = k < 20.0
    assert np.abs(fk[sel] * (k[sel] ** 2 + 1) ** 2 / (8 * np.pi) - 1).max() < 1e-4
    back = model.fourier_bessel(fk, rmax, 1)
    assert np.abs(back - orc.fb_k2r(fk, rmax)).max() < 1e-12 * np.abs(back).max()
    assert np.abs(back - fr).max() < 1e-12


@pytest.mark.parametrize("pot,gam,kap,lam", [("yukawa", 10.0, 1.0, 1.0), ("coulomb", 10.0, 0.0, 1.0),
                                             ("hansen_mcdonald", 0.5, 0.0, 2 * np.sqrt(np.pi * 0.5))])
def test_hnc_matches_oracle(hg, orc, pot, gam, kap, lam):
    n0 = 3 / (4 * np.pi)
    g = hg.hnc_solve(pot, gam, kap, lam, n0, 4096, 60.0, 1e-9, 0.2, 5000)
    o = orc.hnc_solve(orc.make_pot(pot, gam, kap, lam), n0, 4096, 60.0, 1e-9, 0.2, 5000)
    assert g["converged"] and o.converged
    # both iterate to the 1e-9 residual tolerance; the DST summation order differs
    assert np.abs(g["ck"] - o.ck).max() / np.abs(o.ck).max() < 1e-7
    assert abs(g["u_ex"] - o.u_ex) < 1e-7 * abs(o.u_ex)


CASES = {
    "ion_newtonian_3d": dict(ION, nx=16, ny=12, nz=8, lx=20.0, ly=15.0, lz=10.0, closure="newtonian"),
    "ion_maxwell_3d": dict(ION, nx=16, ny=8, nz=12, lx=20.0, ly=10.0, lz=15.0, closure="maxwell",
                           tau_model="constant", tau=1.5),
    "ion_maxwell_ichimaru": dict(ION, nx=12, ny=12, nz=12, lx=15.0, ly=15.0, lz=15.0, gamma=50.0,
                                 kappa=2.0, closure="maxwell", tau_model="ichimaru"),
    "electron_driven_3d": dict(ELEC, nx=16, ny=8, nz=8, lx=20.0, ly=10.0, lz=10.0, closure="newtonian",
                               vext="driven", vext_amplitude=1e-3, vext_mode=(2, 1, 0),
                               vext_omega=0.9, vext_ramp=0.05),
    "ion_1d": dict(ION, nx=32, ny=1, nz=1, lx=20.0, closure="newtonian", gamma=2.0, kappa=0.1,
                   transport="constant", eta=0.3),
    "ion_2d_maxwell": dict(ION, nx=32, ny=4, nz=1, lx=20.0, ly=5.0, closure="maxwell",
                           tau_model="constant", tau=2.0, transport="constant", eta=0.2),
    "ion_nodealias_mode": dict(ION, nx=24, ny=6, nz=6, lx=20.0, ly=5.0, lz=5.0, dealias=False,
                               vext="mode", vext_amplitude=1e-3, vext_mode=(1, 1, 1), eta=0.4,
                               transport="constant"),
    # sizes with register-FFT plans on every axis (32, 48, 64, 96, 256)
    "fast_ion_maxwell_32x48x64": dict(ION, nx=32, ny=48, nz=64, lx=16.0, ly=24.0, lz=32.0,
                                      closure="maxwell", tau_model="constant", tau=1.5),
    "fast_electron_driven_64x96x32": dict(ELEC, nx=64, ny=96, nz=32, lx=20.0, ly=30.0, lz=10.0,
                                          closure="newtonian", vext="driven", vext_amplitude=1e-3,
                                          vext_mode=(3, -1, 1), vext_omega=1.1, vext_ramp=0.0),
    "fast_ion_newtonian_256x8x8": dict(ION, nx=256, ny=8, nz=8, lx=64.0, ly=4.0, lz=4.0,
                                       closure="newtonian"),
    "fast_ion_maxwell_16x16x256": dict(ION, nx=16, ny=16, nz=256, lx=8.0, ly=8.0, lz=64.0,
                                       closure="maxwell", tau_model="constant", tau=0.7),
    # the gaussian external potential (static force from its spectral gradient)
    "ion_gaussian_3d": dict(ION, nx=16, ny=12, nz=8, lx=20.0, ly=15.0, lz=10.0, closure="newtonian",
                            vext="gaussian", vext_amplitude=0.05, vext_width=2.5),
    "fast_ion_gaussian_32x32x32": dict(ION, nx=32, ny=32, nz=32, lx=16.0, ly=16.0, lz=16.0,
                                       closure="newtonian", vext="gaussian", vext_amplitude=0.05,
                                       vext_width=2.0),
    "fast_ion_maxwell_gaussian_32x48x32": dict(ION, nx=32, ny=48, nz=32, lx=16.0, ly=24.0, lz=16.0,
                                               closure="maxwell", tau_model="constant", tau=1.5,
                                               vext="gaussian", vext_amplitude=0.05, vext_width=2.0),
    "electron_gaussian_2d": dict(ELEC, nx=32, ny=16, nz=1, lx=20.0, ly=10.0, closure="newtonian",
                                 vext="gaussian", vext_amplitude=0.02, vext_width=3.0),
    # the transport fits (transport.f90:81-90): Stanton-Murillo ion viscosity
    # and the electron viscosity interpolation
    "ion_stanton_murillo_3d": dict(ION, nx=16, ny=8, nz=8, lx=20.0, ly=10.0, lz=10.0, gamma=2.0, kappa=0.5,
                                   closure="newtonian", transport="stanton_murillo"),
    "ion_stanton_murillo_maxwell": dict(ION, nx=16, ny=12, nz=8, lx=20.0, ly=15.0, lz=10.0, gamma=5.0,
                                        kappa=1.0, closure="maxwell", tau_model="ichimaru",
                                        transport="stanton_murillo"),
    "electron_fit_3d": dict(ELEC, nx=16, ny=8, nz=8, lx=20.0, ly=10.0, lz=10.0, rs=1.86, theta=1.0,
                            closure="newtonian", transport="electron_fit"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_rhs_fp64(hg, orc, case):
    m, o = pair(hg, orc, dt=0.01, **CASES[case])
    n, mom, pi = seeded_state(m)
    m.set_state(n, mom, pi)
    o.set_state(n, mom, pi)
    # the oracle projects nothing: hand it the GPU's dealiased state
    n2, mom2, pi2 = m.get_state()
    assert rel(n2, n) < 1e-12
    o.set_state(n2, mom2, pi2)
    t = 0.37
    dn, dmom, dpi = m.rhs(t)
    on, omom, opi = o.rhs(t)
    assert rel(dn, on) < TOL64, rel(dn, on)
    assert rel(dmom, omom) < TOL64, rel(dmom, omom)
    if m.has_pi:
        assert rel(dpi, opi) < TOL64, rel(dpi, opi)


@pytest.mark.parametrize("case", sorted(CASES))
def test_advance_fp64(hg, orc, case):
    m, o = pair(hg, orc, dt=0.02, **CASES[case])
    n, mom, pi = seeded_state(m)
    m.set_state(n, mom, pi)
    n2, mom2, pi2 = m.get_state()
    o.set_state(n2, mom2, pi2)
    m.advance(5)
    o.advance(5)
    g = m.get_state()
    assert abs(m.t - o.t) < 1e-14 and m.step == 5
    assert rel(g[0], o.n) < TOL64, rel(g[0], o.n)
    assert rel(g[0] - g[0].mean(), o.n - o.n.mean()) < 1e-9
    assert rel(g[1], o.mom) < TOL64, rel(g[1], o.mom)
    if m.has_pi:
        assert rel(g[2], o.pi) < TOL64, rel(g[2], o.pi)


@pytest.mark.parametrize("case", ["ion_newtonian_3d", "ion_maxwell_3d", "electron_driven_3d",
                                  "fast_ion_maxwell_32x48x64", "fast_electron_driven_64x96x32"])
def test_advance_fp32(hg, orc, case):
    m, o = pair(hg, orc, dt=0.02, gpu_precision="fp32", **CASES[case])
    n, mom, pi = seeded_state(m)
    m.set_state(n, mom, pi)
    n2, mom2, pi2 = m.get_state()
    o.set_state(n2, mom2, pi2)
    m.advance(20)
    o.advance(20)
    g = m.get_state()
    assert rel(g[0], o.n) < TOL32
    assert rel(g[1], o.mom) < TOL32, rel(g[1], o.mom)
    if m.has_pi:
        assert rel(g[2], o.pi) < TOL32, rel(g[2], o.pi)


@pytest.mark.parametrize("kind", ["s", "c"])
def test_structure_file_source_matches_oracle(hg, orc, tmp_path, kind):
    """structure = 'file' (structure_source.f90:87-138) with an HNC table
    written as S(k) or c(k): the GPU's c(k) table equals the oracle's read
    of the same file, and rhs / 5-step advance match to 1e-10."""
    n0 = 3.0 / (4.0 * np.pi)
    st = orc.structure_from_hnc(orc.make_pot("yukawa", 10.0, 0.5), n0, 2048, 40.0, 1e-9, 0.2, 5000)
    path = tmp_path / ("table_%s.dat" % kind)
    col = 1.0 / (1.0 - n0 * st.c) if kind == "s" else st.c
    with open(path, "w") as f:
        f.write("# k  %s(k) from HNC\n" % ("S" if kind == "s" else "c"))
        for k, v in zip(st.k, col):
            f.write("%22.14e %22.14e\n" % (k, v))
    kw = dict(kind="ion", gamma=10.0, kappa=0.5, nx=16, ny=8, nz=8, lx=20.0, ly=10.0, lz=10.0,
              transport="yukawa_fit", closure="newtonian", dt=0.02)
    m = hg.Model(hg.default_params(structure="file", structure_file=str(path), structure_kind=kind, **kw))
    so = orc.structure_from_file(str(path), kind, n0)
    k, c = m.structure()
    assert k.size == so.k.size
    assert np.abs(k - so.k).max() <= 1e-15 * so.k.max()
    assert np.abs(c - so.c).max() <= 1e-14 * np.abs(so.c).max()
    o = orc.Model(orc.params(**kw), so)
    n, mom, pi = seeded_state(m)
    m.set_state(n, mom, pi)
    n2, mom2, pi2 = m.get_state()
    o.set_state(n2, mom2, pi2)
    dn, dmom, _ = m.rhs(0.1)
    on, omom, _ = o.rhs(0.1)
    assert rel(dn, on) < TOL64 and rel(dmom, omom) < TOL64
    m.advance(5)
    o.advance(5)
    g = m.get_state()
    assert rel(g[0], o.n) < TOL64 and rel(g[1], o.mom) < TOL64
    m.close()


def test_budgets_and_mode(hg, orc):
    m, o = pair(hg, orc, dt=0.02, **CASES["ion_newtonian_3d"])
    n, mom, _ = seeded_state(m)
    m.set_state(n, mom)
    n2, mom2, _ = m.get_state()
    o.set_state(n2, mom2)
    mass, mm, ek, fe, nmin, nmax = m.budgets()
    omass, omm, oek, ofe = o.budgets()
    assert abs(mass / omass - 1) < 1e-13
    assert np.abs(mm - omm).max() < 1e-13 * omass
    assert abs(ek / oek - 1) < 1e-12
    assert abs(nmin - n2.min()) < 1e-14 and abs(nmax - n2.max()) < 1e-14
    # spec_mode takes mx >= 0 (spectral.f90:179-188); a negative mx is
    # answered with the conjugate of mode (-mx,-my,-mz)
    for (mx, my, mz) in [(1, 0, 0), (2, -1, 3), (0, 2, -2), (-1, 1, 1), (7, 0, 0)]:
        for f, arr in ((0, n2), (1, mom2[0]), (2, mom2[1])):
            ref = o.mode(arr, mx, my, mz) if mx >= 0 else np.conj(o.mode(arr, -mx, -my, -mz))
            assert abs(m.mode(f, mx, my, mz) - ref) < 1e-15 + 1e-12 * abs(ref)


def test_compute_dt_matches_oracle(hg, orc):
    kw = dict(CASES["ion_newtonian_3d"])
    kw.update(dt=0.0, cfl=0.3)
    m, o = pair(hg, orc, **kw)
    n, mom, _ = seeded_state(m)
    m.set_state(n, mom)
    n2, mom2, _ = m.get_state()
    o.set_state(n2, mom2)
    assert abs(m.compute_dt() / o.compute_dt() - 1) < 1e-12


def test_initial_conditions(hg, orc):
    kw = dict(CASES["ion_newtonian_3d"])
    m, o = pair(hg, orc, dt=0.02, **kw)
    for kind in ("mode", "gaussian", "uniform"):
        m.set_initial_condition(kind, 1e-3, (2, 1, 0), 2.0)
        o.set_ic(kind, 1e-3, (2, 1, 0), 2.0)
        assert rel(m.n, o.n) < 1e-13, kind
    m.set_initial_condition("random", 0.02, seed=7)
    d = ic.random_field(16, 12, 8, 20.0, 15.0, 10.0, seed=7)
    assert rel(m.n, m.scalar("n0") * (1 + 0.02 * d)) < 1e-13


def test_set_state_rejects_a_nonpositive_density(hg):
    m = hg.Model(hg.default_params(dt=0.5, **CASES["ion_newtonian_3d"]))
    n = np.full(m.shape, m.scalar("n0"))
    n[3, 2, 1] = 0.0
    with pytest.raises(hg.HydftError) as e:
        m.set_state(n)
    assert e.value.code == 3
    n[3, 2, 1] = np.nan
    with pytest.raises(hg.HydftError) as e:
        m.set_state(n)
    assert e.value.code == 3
    m.close()


def test_nonpositive_density_is_an_error(hg):
    m = hg.Model(hg.default_params(dt=0.5, **CASES["ion_1d"]))
    n0 = m.scalar("n0")
    x = np.arange(32) * 20.0 / 32
    n = n0 * (1 + 0.95 * np.cos(2 * np.pi * x / 20.0)).reshape(1, 1, 32)
    m.set_state(n, np.zeros((3, 1, 1, 32)) + 0.3 * n0)
    with pytest.raises(hg.HydftError) as e:
        m.advance(50)
    assert e.value.code in (3, 4)


ENERGY_CASES = ["ion_newtonian_3d", "ion_maxwell_ichimaru", "electron_driven_3d", "ion_nodealias_mode",
                "ion_gaussian_3d", "fast_ion_maxwell_gaussian_32x48x32", "electron_gaussian_2d", "ion_1d"]


@pytest.mark.parametrize("case", ENERGY_CASES)
def test_free_energy_matches_oracle(hg, orc, case):
    """budgets' F (functional_t%energy + the external potential as last
    evaluated, diagnostics.f90:41-60) against the oracle, before and after
    steps."""
    m, o = pair(hg, orc, dt=0.01, **CASES[case])
    n, mom, pi = seeded_state(m)
    m.set_state(n, mom, pi)
    o.set_state(n, mom, pi)
    fe = m.budgets()[3]
    ofe = o.budgets()[3]
    assert abs(fe - ofe) <= TOL64 * max(abs(ofe), 1e-300)
    m.advance(3)
    o.advance(3)
    fe = m.budgets()[3]
    ofe = o.budgets()[3]
    assert abs(fe - ofe) <= TOL64 * max(abs(ofe), 1e-300)


def test_tile_shapes_give_identical_results(hg, monkeypatch):
    """The autotuner's candidate tile shapes (kx columns per y/z block, threads
    per x block) only change the blocking: every shape gives the same fields
    to the bit, and the tuned model keeps one of the candidates."""
    kw = dict(ION, nx=64, ny=32, nz=48, lx=32.0, ly=16.0, lz=24.0, closure="maxwell", tau_model="constant",
              tau=1.5, dt=0.01, gpu_precision="fp32")
    out = []
    for tile, nt in (("8", "128"), ("16", "256"), ("8", "256"), ("32", "256")):
        monkeypatch.setenv("HYDFT_YZ_TILE", tile)
        monkeypatch.setenv("HYDFT_X_THREADS", nt)
        m = hg.Model(hg.default_params(**kw))
        n, mom, pi = seeded_state(m)
        m.set_state(n, mom, pi)
        m.advance(3)
        assert m.scalar("yz_tile") == int(tile) and m.scalar("x_threads") == int(nt)
        out.append(m.get_state())
        m.close()
    for other in out[1:]:
        for x, y in zip(out[0], other):
            assert np.array_equal(x, y)
    monkeypatch.delenv("HYDFT_YZ_TILE")
    monkeypatch.delenv("HYDFT_X_THREADS")
    m = hg.Model(hg.default_params(**kw))
    n, mom, pi = seeded_state(m)
    m.set_state(n, mom, pi)
    m.advance(3)
    assert m.scalar("yz_tile") in (8, 16, 32) and m.scalar("x_threads") in (128, 256)
    assert m.scalar("yz_tile_fwd") in (8, 16, 32)
    for x, y in zip(m.get_state(), out[0]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_tma_tile_loads_give_identical_results(hg, monkeypatch, prec):
    """The y inverse, y forward and z forward passes of a 128^3 model (which
    steps with the plain kernels) read their input tiles with TMA tensor
    loads, and with HYDFT_TMA_ZINV=1 the z inverse pass too; with
    HYDFT_TMA_YST / _YFST / _ZFST / _ZIST = 1 the y inverse, y forward,
    z forward and (one row per thread) z inverse passes write their output
    tiles with tensor stores; with
    HYDFT_TMA=0 every thread loads its own elements.  Same fields to the
    bit, after steps and in the right-hand side."""
    kw = dict(ION, nx=128, ny=128, nz=128, lx=64.0, ly=64.0, lz=64.0, closure="maxwell", tau_model="constant",
              tau=1.5, dt=0.01, gpu_precision=prec)
    names = ("HYDFT_TMA", "HYDFT_TMA_ZINV", "HYDFT_TMA_YST", "HYDFT_TMA_YFST", "HYDFT_TMA_ZFST", "HYDFT_TMA_ZIST",
             "HYDFT_ZNB")
    configs = [("0", "0", "0", "0", "0", "0", "2"),   # per-thread loads and stores
               ("1", "1", "1", "1", "1", "0", "2"),   # tensor loads (z inverse too), tensor stores
               ("1", "0", "1", "1", "1", "1", "1"),   # one row per thread in the z inverse, its tensor store
               ("1", "1", "1", "1", "1", "1", "1")]   # ... and its tensor load
    out = []
    for cfg in configs:
        for name, val in zip(names, cfg):
            monkeypatch.setenv(name, val)
        m = hg.Model(hg.default_params(**kw))
        n, mom, pi = seeded_state(m, seed=9)
        m.set_state(n, mom, pi)
        r = m.rhs(0.2)
        m.advance(3)
        out.append(list(m.get_state()) + list(r))
        m.close()
    for name in names:
        monkeypatch.delenv(name)
    for fields in zip(*out):
        if fields[0] is not None:
            for other in fields[1:]:
                assert np.array_equal(fields[0], other)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_band_classified_passes_match_runtime_band_test(hg, monkeypatch, prec):
    """With the two-thirds band limit M = (L - 1) / 3 the register-FFT passes
    classify the band elements at compile time and skip the ones outside
    the band; the fields equal those of the passes that test every element
    at run time (HYDFT_BAND=0).  Without dealiasing no axis qualifies."""
    kw = dict(ION, nx=64, ny=32, nz=48, lx=32.0, ly=16.0, lz=24.0, closure="maxwell", tau_model="constant",
              tau=1.5, dt=0.01, gpu_precision=prec)
    out = []
    for flag, axes in (("0", 0), ("1", 7)):
        monkeypatch.setenv("HYDFT_BAND", flag)
        m = hg.Model(hg.default_params(**kw))
        assert m.scalar("band_axes") == axes
        n, mom, pi = seeded_state(m)
        m.set_state(n, mom, pi)
        m.advance(3)
        out.append(m.get_state())
        m.close()
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)
    monkeypatch.delenv("HYDFT_BAND")
    m = hg.Model(hg.default_params(**dict(kw, dealias=False)))
    assert m.scalar("band_axes") == 0
    m.close()


@pytest.mark.parametrize("prec,base", [("fp32", 256), ("fp64", 128)])
def test_wide_yz_blocks_give_identical_results(hg, monkeypatch, prec, base):
    """On 256-point y and z axes the autotuner also tries y/z blocks of twice
    the threads (two rows of the other axis, or 32 kx columns, per block);
    they give the same fields to the bit as the narrow blocks."""
    kw = dict(ION, nx=32, ny=256, nz=256, lx=16.0, ly=128.0, lz=128.0, closure="maxwell", tau_model="constant",
              tau=1.5, dt=0.01, gpu_precision=prec)
    out = []
    for tile, nt in (("16", base), ("16", 2 * base), ("8", 2 * base), ("32", base)):
        monkeypatch.setenv("HYDFT_YZ_TILE", tile)
        monkeypatch.setenv("HYDFT_YZ_THREADS", str(nt))
        m = hg.Model(hg.default_params(**kw))
        n, mom, pi = seeded_state(m)
        m.set_state(n, mom, pi)
        m.advance(2)
        assert m.scalar("yz_tile") == int(tile) and m.scalar("yz_threads") == nt
        assert m.scalar("yz_tile_fwd") == int(tile) and m.scalar("yz_threads_fwd") == nt
        out.append(m.get_state())
        m.close()
    for other in out[1:]:
        for x, y in zip(out[0], other):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_z_pass_row_pairs_give_identical_results(hg, monkeypatch, prec):
    """The z passes can transform two ky rows per thread (both columns loaded
    before the first is transformed; the inverse pass does in the ensemble
    forms, and both with HYDFT_ZNB=2 / HYDFT_ZNB_FWD=2); the fields equal
    those of one row per thread in both passes (the inverse one then writing
    its output tiles with tensor stores) to the bit."""
    kw = dict(ION, nx=64, ny=32, nz=48, lx=32.0, ly=16.0, lz=24.0, closure="maxwell", tau_model="constant",
              tau=1.5, dt=0.01, gpu_precision=prec)
    out = []
    for flag in ("1", "2"):
        monkeypatch.setenv("HYDFT_ZNB", flag)
        monkeypatch.setenv("HYDFT_ZNB_FWD", flag)
        m = hg.Model(hg.default_params(**kw))
        n, mom, pi = seeded_state(m)
        m.set_state(n, mom, pi)
        m.advance(3)
        out.append(m.get_state())
        m.close()
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_tuned_radix_plans_match_oracle(hg, orc, monkeypatch, prec, tol):
    """Axes without a register plan (72, 36, 24 here) run the generic
    Stockham passes, whose radix sequence the autotuner picks: it times the
    phase-B transforms with the 2^a part in radix-8 or radix-4 steps, either
    order, the radix-3 steps first or last, and keeps the fastest (the
    scalars radix_x/y/z give the chosen sequence as digits, positive when
    the tuner chose it).  Whichever it keeps, five Maxwell steps match the
    oracle."""
    monkeypatch.delenv("HYDFT_RADIX", raising=False)
    kw = dict(ION, nx=72, ny=36, nz=24, lx=36.0, ly=18.0, lz=12.0, closure="maxwell", tau_model="constant",
              tau=1.5, dt=0.02, gpu_precision=prec)
    m, o = pair(hg, orc, **kw)
    n, mom, pi = seeded_state(m)
    m.set_state(n, mom, pi)
    n2, mom2, pi2 = m.get_state()
    o.set_state(n2, mom2, pi2)
    m.advance(5)
    o.advance(5)
    for ax, L in (("radix_x", 72), ("radix_y", 36), ("radix_z", 24)):
        code = int(m.scalar(ax))
        assert code > 0
        assert int(np.prod([int(d) for d in str(code)])) == L
    g = m.get_state()
    assert rel(g[0], o.n) < tol, rel(g[0], o.n)
    assert rel(g[1], o.mom) < tol, rel(g[1], o.mom)
    assert rel(g[2], o.pi) < tol, rel(g[2], o.pi)
