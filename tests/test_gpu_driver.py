"""The driver loop (hydft_gpu_run) and the .bin field files.

run() follows src/hydft.f90:30-60 and writes <prefix>_diag.dat and
<prefix>_probe.dat as diagnostics.f90 does; the same loop written here over
the oracle (FP64, the reference's algorithm) gives the numbers the files must
hold.  The field files follow io.f90:19-35; the reader below restates
python/hydft_io.py:45-56.
"""
import numpy as np
import pytest

from hydft_b200 import ic

pytestmark = pytest.mark.gpu

HNC = dict(hnc_nr=2048, hnc_rmax=40.0)


@pytest.fixture(scope="module")
def hg():
    import hydft_b200
    hydft_b200.lib()
    return hydft_b200


def read_bin(path):
    with open(path, "rb") as f:
        nx, ny, nz, ndim, npi = np.fromfile(f, dtype=np.int32, count=5)
        t, lx, ly, lz = np.fromfile(f, dtype=np.float64, count=4)
        n = np.fromfile(f, dtype=np.float64, count=nx * ny * nz).reshape((nz, ny, nx))
        mom = np.fromfile(f, dtype=np.float64, count=3 * nx * ny * nz).reshape((3, nz, ny, nx))
        pi = None
        if npi > 0:
            pi = np.fromfile(f, dtype=np.float64, count=npi * nx * ny * nz).reshape((npi, nz, ny, nx))
        rest = f.read()
    return dict(nx=nx, ny=ny, nz=nz, ndim=ndim, npi=npi, t=t, lx=lx, ly=ly, lz=lz, n=n, mom=mom, pi=pi,
                rest=rest)


def seeded(m, seed):
    p = m.p
    n0 = m.scalar("n0")
    n = n0 * (1 + 0.01 * ic.random_field(m.nx, m.ny, m.nz, p.lx, p.ly, p.lz, seed))
    mom = np.zeros((3,) + m.shape)
    mom[0] = 0.004 * n0 * ic.random_field(m.nx, m.ny, m.nz, p.lx, p.ly, p.lz, seed + 1)
    pi = None
    if m.has_pi:
        pi = np.zeros((6,) + m.shape)
        pi[3] = 1e-3 * ic.random_field(m.nx, m.ny, m.nz, p.lx, p.ly, p.lz, seed + 2)
    return n, mom, pi


@pytest.mark.parametrize("closure", ["newtonian", "maxwell"])
def test_field_files_round_trip_and_resume(hg, tmp_path, closure):
    kw = dict(kind="ion", gamma=10.0, kappa=1.0, transport="yukawa_fit", nx=16, ny=12, nz=8, lx=20.0, ly=15.0,
              lz=10.0, closure=closure, tau_model="constant", tau=1.5, dt=0.01, **HNC)
    m = hg.Model(hg.default_params(**kw))
    m.set_state(*seeded(m, 3))
    m.advance(4)
    prefix = str(tmp_path / "run")
    m.write_fields(prefix)
    path = tmp_path / "run_fld_000004.bin"
    d = read_bin(path)
    n, mom, pi = m.get_state()
    assert (d["nx"], d["ny"], d["nz"], d["ndim"]) == (16, 12, 8, 3)
    assert d["npi"] == (6 if closure == "maxwell" else 0) and d["rest"] == b""
    assert d["t"] == m.t and (d["lx"], d["ly"], d["lz"]) == (20.0, 15.0, 10.0)
    assert np.array_equal(d["n"], n) and np.array_equal(d["mom"], mom)
    if pi is not None:
        assert np.array_equal(d["pi"], pi)
    # resume: a fresh model read from the file continues as the original
    r = hg.Model(hg.default_params(**kw))
    r.read_fields(path)
    assert r.step == 4 and r.t == m.t
    r2 = r.get_state()
    # the state goes back through a forward and an inverse transform
    assert np.abs(r2[0] - n).max() <= 1e-13 * np.abs(n).max()
    assert np.abs(r2[1] - mom).max() <= 1e-13 * np.abs(n).max()
    m.advance(3)
    r.advance(3)
    a, b = m.get_state(), r.get_state()
    for x, y in zip(a, b):
        if x is not None:
            assert np.abs(x - y).max() <= 1e-12 * np.abs(x).max()
    m.close()
    r.close()


def test_read_fields_rejects_another_grid(hg, tmp_path):
    kw = dict(kind="ion", gamma=10.0, kappa=1.0, nx=16, ny=12, nz=8, lx=20.0, ly=15.0, lz=10.0, dt=0.01, **HNC)
    m = hg.Model(hg.default_params(**kw))
    m.write_fields(str(tmp_path / "a"))
    other = hg.Model(hg.default_params(**dict(kw, nx=32)))
    with pytest.raises(hg.HydftError):
        other.read_fields(tmp_path / "a_fld_000000.bin")


def parse(path):
    rows = [ln.split() for ln in open(path) if not ln.startswith("#")]
    return np.array([[float(x.replace("D", "E")) for x in r] for r in rows])


def oracle_run(hg, orc, kw, state, p):
    """hydft_run's loop (src/hydft.f90:30-60) over the oracle."""
    g = hg.Model(hg.default_params(**kw))
    k, c = g.structure()
    st = orc.Structure(k, c, g.scalar("n0"), g.scalar("u_ex"), g.scalar("du_dgamma"), True)
    n0 = g.scalar("n0")
    g.close()
    drop = {"gpu_precision", "prefix", "tend", "nsteps_max", "iprobe", "idiag", "iout", "probe_mode"}
    okw = {kk: v for kk, v in kw.items() if kk not in drop}
    o = orc.Model(orc.params(**okw), st)
    o.set_state(*state)
    diag, probe = [], []

    def d():
        mass, mom, ek, fe = o.budgets()
        n = o.n
        diag.append([o.step, o.t, o.dt, mass, *mom, ek, fe, ek + fe, n.min(), n.max()])

    def pr():
        a = o.mode(o.n, *p["probe_mode"]) / n0
        b = o.mode(o.mom[0], *p["probe_mode"])
        probe.append([o.t, a.real, a.imag, abs(a), b.real, b.imag])

    o.compute_dt()
    d()
    pr()
    irec = 0
    while o.t < p["tend"] and o.step < p["nsteps_max"]:
        if irec == 0:
            o.compute_dt()
        irec = (irec + 1) % 20
        if o.t + o.dt > p["tend"]:
            o.set("dt", p["tend"] - o.t)
        o.advance(1)
        if o.step % p["iprobe"] == 0:
            pr()
        if o.step % p["idiag"] == 0:
            d()
    if o.step % p["idiag"] != 0:
        d()
    return np.array(diag), np.array(probe)


def test_run_matches_the_reference_loop(hg, orc, tmp_path):
    prefix = str(tmp_path / "drv")
    run = dict(tend=1.23, nsteps_max=100000, iprobe=2, idiag=7, iout=0, probe_mode=(1, 0, 0))
    kw = dict(kind="ion", gamma=10.0, kappa=1.0, transport="yukawa_fit", nx=16, ny=12, nz=8, lx=20.0,
              ly=15.0, lz=10.0, closure="newtonian", dt=0.0, cfl=0.4, prefix=prefix, vext="driven",
              vext_amplitude=1e-3, vext_mode=(1, 0, 0), vext_omega=0.8, **HNC, **run)
    m = hg.Model(hg.default_params(**kw))
    state = seeded(m, 11)
    m.set_state(*state)
    # about 45 steps: three dt updates and a shortened last step
    run["tend"] = 45.37 * m.compute_dt()
    m.close()
    kw.update(run)
    m = hg.Model(hg.default_params(**kw))
    m.set_state(*state)
    m.run()
    diag, probe = parse(prefix + "_diag.dat"), parse(prefix + "_probe.dat")
    odiag, oprobe = oracle_run(hg, orc, kw, state, run)
    assert diag.shape == odiag.shape and probe.shape == oprobe.shape
    assert diag.shape[0] > 5 and probe.shape[0] > 20
    assert np.array_equal(diag[:, 0], odiag[:, 0])                  # step numbers
    assert abs(diag[-1, 1] - run["tend"]) < 1e-9 * run["tend"]     # ends at tend (10 digits in the file)
    # the files hold 10 significant digits
    assert np.allclose(diag[:, 1:], odiag[:, 1:], rtol=2e-9, atol=1e-12)
    assert np.allclose(probe, oprobe, rtol=2e-9, atol=1e-15)
    header = open(prefix + "_probe.dat").readline()
    assert header.startswith("# probe mode   1   0   0:")
    m.close()


def test_run_writes_field_files(hg, tmp_path):
    prefix = str(tmp_path / "out")
    kw = dict(kind="ion", gamma=10.0, kappa=1.0, nx=16, ny=12, nz=8, lx=20.0, ly=15.0, lz=10.0, dt=0.02,
              tend=0.2, iout=4, idiag=5, iprobe=1, prefix=prefix, **HNC)
    m = hg.Model(hg.default_params(**kw))
    m.set_initial_condition("mode", 1e-3, (1, 0, 0))
    m.run()
    names = sorted(p.name for p in tmp_path.glob("out_fld_*.bin"))
    assert names == ["out_fld_%06d.bin" % s for s in (0, 4, 8)]
    # ten steps of 0.02 end just short of 0.2 in FP64; the eleventh is cut to end at tend
    assert m.step == 11 and m.t == 0.2
    d = read_bin(tmp_path / "out_fld_000008.bin")
    assert abs(d["t"] - 0.16) < 1e-12
    m.close()
