"""The driven chi(k, w) measurement of the C3 configuration on the GPU path,
against the oracle's linear response (linear_response.f90:72-76) with the
reference's threshold (test/test_driven_mode.f90:62-64: 2 % on chi, 5 % on
the transient scatter).

Electrons r_s = 1, theta = 1 (Thomas-Fermi, gradient, Hartree, RY terms),
128^3 box of L = 40, constant eta = 0.2, v_ext = 1e-4 cos(q.x - w t) at
q = 2 pi/L (3, 0, 0), 4000 RK3 steps from the uniform state, dt from
compute_dt at cfl 0.8.  Eight drive frequencies spread over [0.5, 3] w_p
(every fourth of the 32-point sweep that bench.py --workload chi runs)
advance as one ensemble in FP32; two of them also in FP64, and the
FP32 fields must stay within 1e-5 of the FP64 ones after the 4000 steps.
chi is read from the steady response as the reference's fit does: the mean
of n(k, t) e^{i w t} over the last 40 % of the run, times 2/A.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, L, MODE, AMP, STEPS, EVERY = 128, 40.0, 3, 1e-4, 4000, 10
OMEGAS = np.linspace(0.5, 3.0, 32)[::4]


@pytest.fixture(scope="module")
def hg():
    import hydft_b200
    hydft_b200.lib()
    return hydft_b200


def member(w, precision):
    return dict(kind="electron", rs=1.0, theta=1.0, nx=N, ny=N, nz=N, lx=L, ly=L, lz=L, closure="newtonian",
                transport="constant", eta=0.2, vext="driven", vext_amplitude=AMP, vext_mode=(MODE, 0, 0),
                vext_omega=float(w), hnc_nr=4096, hnc_rmax=80.0, cfl=0.8, dt=0.0, gpu_precision=precision)


def run(hg, omegas, precision):
    b = hg.Batch([hg.default_params(**member(w, precision)) for w in omegas])
    try:
        dts = []
        for m in b.members:
            m.set_state(np.full((N, N, N), m.scalar("n0")))
            dts.append(m.compute_dt())
        dt = min(dts)
        for m in b.members:
            m.set_time(0.0, dt)
        ts, zs = [], [[] for _ in omegas]
        for k in range(STEPS // EVERY):
            b.advance(EVERY)
            ts.append((k + 1) * EVERY * dt)
            for i, m in enumerate(b.members):
                zs[i].append(m.mode(0, MODE, 0, 0))
        groups = b.grouped()
        states = [m.get_state() for m in b.members]
        return np.array(ts), [np.array(z) for z in zs], states, groups, dt
    finally:
        b.close()


def test_driven_chi_sweep_matches_linear_response(hg, orc):
    ts, zs, states, groups, dt = run(hg, OMEGAS, "fp32")
    assert abs(ts[-1] - STEPS * dt) < 1e-9 * ts[-1]
    # the oracle's linear response of the same electron fluid (the same
    # functional, transport and closure; the response does not depend on
    # the box's y and z extent)
    o = orc.Model(orc.params(kind="electron", rs=1.0, theta=1.0, nx=N, ny=1, nz=1, lx=L, closure="newtonian",
                             transport="constant", eta=0.2, hnc_nr=4096, hnc_rmax=80.0))
    q = 2.0 * np.pi * MODE / L
    errs = []
    for w, z in zip(OMEGAS, zs):
        a, scatter = orc.fit_driven_response(ts, z, w, 0.6 * ts[-1])
        chi_sim = 2.0 * a / AMP
        chi_lin = o.chi(q, w)
        errs.append(abs(chi_sim - chi_lin) / abs(chi_lin))
        assert errs[-1] < 0.02, (w, errs[-1])
        assert scatter < 0.05, (w, scatter)
    print("chi sweep, relative error per drive frequency:", dict(zip(np.round(OMEGAS, 3), np.round(errs, 5))))
    # FP32 against FP64 after the 4000 steps, at one frequency below and one
    # near the mode's resonance
    pick = [0, 2]
    _, _, s64, _, dt64 = run(hg, OMEGAS[pick], "fp64")
    assert abs(dt64 - dt) <= 1e-12 * dt
    for j, i in enumerate(pick):
        a, b = states[i], s64[j]
        for x, y in ((a[0], b[0]), (a[1], b[1])):
            assert np.linalg.norm(x - y) / np.linalg.norm(y) < 1e-5
