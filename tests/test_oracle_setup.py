"""The reference's setup-path tests restated against the oracle, with their
thresholds: test/test_transport.f90 (Stanton-Murillo fits and the electron
viscosity), test/test_structure_file.f90 (the file structure source) and
test/test_dispersion.f90 (the linear theory the GPU physics tests use as
their truth).

test_transport.f90's binary-mixture checks (sm_mixture) are not restated:
the solver step never calls the mixture formulas, and the oracle does not
carry them.
"""
import numpy as np
import pytest

# Table I of PRE 93, 043203 as test_transport.f90:19-26 lists it: D* from MD
# for kappa in KAP (columns) and Gamma in GAM (rows)
KAP = [0.5, 1.0, 1.5, 2.0]
GAM = [0.1, 0.3, 0.5, 0.7, 1.0, 2.0, 5.0]
DMD = np.array([
    [143.0, 16.4, 6.4, 3.76, 2.14, 0.82, 0.28],
    [173.0, 20.9, 8.41, 4.72, 2.54, 1.02, 0.31],
    [209.0, 24.5, 10.0, 5.92, 3.15, 1.19, 0.356],
    [241.0, 28.4, 12.3, 7.32, 3.72, 1.52, 0.504]]).T


def test_sm_fits_continuous_at_g_1(orc):
    # test_transport.f90:29-36
    for idx in range(1, 5):
        kl = orc.sm_knm(idx, 1.0 - 1e-12)
        kr = orc.sm_knm(idx, 1.0 + 1e-12)
        assert abs(kl / kr - 1.0) < 5e-3
    assert abs(orc.sm_knm(4, 1.0) - 0.32237) < 1e-4
    assert abs(orc.sm_knm(1, 1e-6) / (-0.25 * np.log(1.4660e-6)) - 1.0) < 1e-4


def test_sm_self_diffusion_against_md_table(orc):
    # test_transport.f90:38-50: within 25 % for Gamma <= 2, 35 % at Gamma = 5
    for j, kap in enumerate(KAP):
        for i, gam in enumerate(GAM):
            err = abs(orc.sm_diffusion(gam, kap) / DMD[i, j] - 1.0)
            assert err < (0.25 if gam <= 2.0 else 0.35), (gam, kap, err)


def test_sm_conductivity_over_viscosity(orc):
    # test_transport.f90:52
    assert abs(orc.sm_conductivity(1.5, 0.7) / orc.sm_viscosity(1.5, 0.7) - 3.75) < 1e-12


def electron_units(orc, rs, gamma):
    """units_t%init('electron', gamma, 0, rs, 1) through a tiny oracle model
    (theta is derived, not given: the model takes gamma as it is)."""
    p = orc.params(kind="electron", rs=rs, gamma=gamma, nx=4, ny=1, nz=1, lx=4.0, terms="tf",
                   structure="none", transport="constant", eta=0.0)
    return orc.Model(p)


def test_electron_viscosity_and_screening_length(orc):
    # test_transport.f90:71-80: r_s = 1.86, Gamma = 1 -> lambda_TF = 0.6472,
    # eta_l = 1.312, eta_CV = 0.00467
    m = electron_units(orc, 1.86, 1.0)
    ltf = m.get("lambda_tf")
    assert abs(ltf - 0.6472) < 5e-4
    eta_l, eta_cv, _ = orc.sm_electron_viscosity(1.86, 1.0, m.get("theta"), ltf)
    assert abs(eta_l - 1.312) < 3e-3
    assert abs(eta_cv - 0.00467) < 2e-5
    # test_transport.f90:82-84: classical limit of lambda_TF is the Debye
    # length 1/sqrt(3 Gamma)
    m = electron_units(orc, 1.0, 0.01)
    assert abs(m.get("lambda_tf") * np.sqrt(3.0 * 0.01) - 1.0) < 5e-3


def test_model_transport_uses_the_fits(orc):
    """transport.f90:81-90: stanton_murillo gives eta = eta*(Gamma, kappa) and
    electron_fit eta_l of sm_electron_viscosity (eta = 3 eta_l/4, xi = 0)."""
    p = orc.params(kind="ion", gamma=2.0, kappa=0.5, nx=4, ny=1, nz=1, lx=4.0, terms="ideal,hartree",
                   structure="none", transport="stanton_murillo")
    m = orc.Model(p)
    assert abs(m.get("eta") - orc.sm_viscosity(2.0, 0.5)) < 1e-14 * orc.sm_viscosity(2.0, 0.5)
    p = orc.params(kind="electron", rs=1.86, gamma=1.0, nx=4, ny=1, nz=1, lx=4.0, terms="tf",
                   structure="none", transport="electron_fit")
    m = orc.Model(p)
    eta_l, _, _ = orc.sm_electron_viscosity(1.86, 1.0, m.get("theta"), m.get("lambda_tf"))
    assert abs(m.get("eta_l") - eta_l) < 1e-14 * eta_l


def test_structure_file_source_reproduces_hnc(orc, tmp_path):
    # test_structure_file.f90:20-41: Yukawa Gamma = 10, kappa = 0.5 HNC
    # written as S(k) (with a comment line) and as c(k), read back; c(k)
    # of both file sources equals the HNC source's to 1e-6 on 200 points
    n0 = 3.0 / (4.0 * np.pi)
    pot = orc.make_pot("yukawa", 10.0, 0.5)
    st = orc.structure_from_hnc(pot, n0, 4096, 60.0, 1e-9, 0.2, 5000)
    s_of_k = 1.0 / (1.0 - n0 * st.c)
    fs = tmp_path / "sk.dat"
    fc = tmp_path / "ck.dat"
    with open(fs, "w") as f:
        f.write("# k  S(k) from HNC\n")
        for k, s in zip(st.k, s_of_k):
            f.write("%22.12e%22.12e\n" % (k, s))
    with open(fc, "w") as f:
        for k, c in zip(st.k, st.c):
            f.write("%22.12e%22.12e\n" % (k, c))
    sf = orc.structure_from_file(str(fs), "s", n0)
    sc = orc.structure_from_file(str(fc), "c", n0)
    emax = 0.0
    for i in range(1, 201):
        q = 0.1 + 0.05 * i
        emax = max(emax, abs(sf.c_of_k(q) - st.c_of_k(q)), abs(sc.c_of_k(q) - st.c_of_k(q)))
    assert emax < 1e-6


def test_structure_file_rejects_bad_tables(orc, tmp_path):
    # structure_source.f90:118,133-137
    f = tmp_path / "bad.dat"
    f.write_text("1.0 0.5\n")
    with pytest.raises(ValueError):
        orc.structure_from_file(str(f), "c", 0.2)
    f.write_text("1.0 0.5\n0.5 0.4\n")
    with pytest.raises(ValueError):
        orc.structure_from_file(str(f), "c", 0.2)
    f.write_text("0.0 0.5\n0.5 0.4\n")
    with pytest.raises(ValueError):
        orc.structure_from_file(str(f), "c", 0.2)


@pytest.fixture(scope="module")
def yukawa_linear(orc):
    """test_dispersion.f90:27-33: Yukawa Gamma = 2, kappa = 0.1, 16 x 1 x 1,
    L = 20, HNC nr 4096 rmax 60, eta 0.3, xi 0.05, Maxwell with constant tau 2."""
    n0 = 3.0 / (4.0 * np.pi)
    st = orc.structure_from_hnc(orc.make_pot("yukawa", 2.0, 0.1), n0, 4096, 60.0, 1e-9, 0.2, 5000)
    kw = dict(kind="ion", gamma=2.0, kappa=0.1, nx=16, ny=1, nz=1, lx=20.0, hnc_nr=4096, hnc_rmax=60.0,
              transport="constant", eta=0.3, xi=0.05, closure="maxwell", tau_model="constant", tau=2.0)
    return st, kw


def test_dispersion_yukawa_maxwell(orc, yukawa_linear):
    # test_dispersion.f90:34-55
    st, kw = yukawa_linear
    m = orc.Model(orc.params(**kw), st)
    eta_bar = m.get("eta_l") / m.get("mass")
    assert abs(eta_bar - (4.0 * 0.3 / 3.0 + 0.05)) < 1e-14
    beta, tau = m.get("beta"), 2.0
    for i in range(1, 6):
        q = 0.4 * i
        sq = st.s_of_k(q)
        assert abs(m.c2(q) * beta * sq - 1.0) < 1e-10
        w = m.dispersion(q)
        # PRE Eq. 54
        res = w * w - q * q / (3.0 * 2.0 * sq) + 1j * eta_bar * q * q * w / (1.0 - 1j * w * tau)
        assert abs(res) < 1e-12
        assert w.real > 0.0 and w.imag < 0.0
        # the root satisfies the cubic (the denominator times 1 - i w tau)
        den = -w * w + q * q * m.c2(q) - 1j * q * q * eta_bar * w / (1.0 - 1j * w * tau)
        assert abs(den * (1.0 - 1j * w * tau)) < 1e-10


def test_dispersion_newtonian_limit_and_static_response(orc, yukawa_linear):
    # test_dispersion.f90:57-73
    st, kw = yukawa_linear
    m = orc.Model(orc.params(**dict(kw, closure="newtonian")), st)
    eta_bar = m.get("eta_l") / m.get("mass")
    q = 1.0
    nu = q * q * eta_bar
    wns = -0.5j * nu + np.sqrt(complex(q * q * m.c2(q) - 0.25 * nu * nu, 0.0))
    assert abs(m.dispersion(q) - wns) < 1e-12
    assert abs(m.chi(q, 0.0).real + 1.0 / m.kernel(q)) < 1e-10
    assert abs(m.dsf(q, 0.7) - m.dsf(q, -0.7)) < 1e-14
    assert m.dsf(q, 0.7) > 0.0


def test_dispersion_electrons(orc):
    # test_dispersion.f90:75-110
    base = dict(kind="electron", rs=1.86, gamma=1.0, nx=16, ny=1, nz=1, lx=20.0, terms="tf,hartree",
                structure="none", transport="constant", eta=0.0, xi=0.0, closure="newtonian")
    m = orc.Model(orc.params(**base))
    n0 = m.get("n0")
    for i in range(1, 5):
        q = 0.5 * i
        w = m.dispersion(q)
        assert abs(w * w - q * q * m.c2(q)) < 1e-12
        assert abs(w.imag) < 1e-12
        assert abs(w.real ** 2 - (1.0 + q * q * n0 * m.term_kernel(0, q))) < 1e-12
    # classical limit: Bohm-Gross w^2 = 1 + q^2/(3 Gamma)
    m = orc.Model(orc.params(**dict(base, gamma=0.01)))
    q = 1.0
    assert abs(m.dispersion(q).real / np.sqrt(1.0 + q * q / (3.0 * 0.01)) - 1.0) < 5e-3
    # detailed balance of the quantum DSF, with viscosity
    m = orc.Model(orc.params(**dict(base, eta=0.2)))
    x = 0.8
    lhs = m.dsf(q, -x)
    rhs = np.exp(-m.get("beta") * m.get("hbar") * x) * m.dsf(q, x)
    assert abs(lhs - rhs) / m.dsf(q, x) < 1e-12
    assert m.dsf(q, x) > 0.0
