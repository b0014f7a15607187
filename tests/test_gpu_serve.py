"""Serving (hydft_serve_*): requests admitted while others run give the same
fields as each model solved alone, admission respects the HBM budget, and
failures reach the caller.

Each request runs on its own stream and the kernels are deterministic, so a
request solved in the mix agrees with the model solved alone to the last
bit.
"""
import numpy as np
import pytest

from hydft_b200 import ic

pytestmark = pytest.mark.gpu

HNC = dict(hnc_nr=2048, hnc_rmax=40.0)
REQUESTS = [
    (dict(kind="ion", gamma=10.0, kappa=1.0, transport="yukawa_fit", nx=32, ny=32, nz=32,
          lx=20.0, ly=20.0, lz=20.0, dt=0.01, gpu_precision="fp32", **HNC), 40, "mode"),
    (dict(kind="ion", gamma=30.0, kappa=2.0, closure="maxwell", transport="yukawa_fit", tau_model="ichimaru",
          nx=32, ny=16, nz=16, lx=16.0, ly=8.0, lz=8.0, gpu_precision="fp32", **HNC), 25, "random"),
    (dict(kind="electron", rs=1.0, theta=1.0, transport="constant", eta=0.2, nx=16, ny=16, nz=16,
          lx=12.0, ly=12.0, lz=12.0, vext="driven", vext_amplitude=1e-3, vext_mode=(1, 0, 0), vext_omega=1.0,
          **HNC), 30, "random"),
    (dict(kind="ion", gamma=10.0, kappa=1.0, transport="yukawa_fit", nx=48, ny=48, nz=48,
          lx=30.0, ly=30.0, lz=30.0, gpu_precision="fp32", **HNC), 35, "random"),
]


@pytest.fixture(scope="module")
def hg():
    import hydft_b200
    hydft_b200.lib()
    return hydft_b200


def params(hg, kw, how):
    extra = dict(ic="mode", ic_amplitude=1e-3, ic_mode=(1, 1, 0)) if how == "mode" else {}
    return hg.default_params(**kw, **extra)


def initial(hg, p, i):
    """A seeded initial state of the model of p (None: p's own IC)."""
    m = hg.Model(p)
    n0 = m.scalar("n0")
    m.close()
    n = n0 * (1 + 0.01 * ic.random_field(p.nx, p.ny, p.nz, p.lx, p.ly, p.lz, 70 + i))
    mom = np.zeros((3, p.nz, p.ny, p.nx))
    mom[0] = 0.004 * n0 * ic.random_field(p.nx, p.ny, p.nz, p.lx, p.ly, p.lz, 80 + i)
    return n, mom, None


def alone(hg, p, nsteps, st):
    m = hg.Model(p)
    if st is None:
        m.set_initial_condition("mode", p.ic_amplitude, tuple(p.ic_mode))
    else:
        m.set_state(st[0], st[1])
    if not p.dt > 0:
        m.compute_dt()
    m.advance(nsteps)
    out = m.get_state(), m.step, m.t
    m.close()
    return out


def test_requests_same_alone_and_in_the_mix(hg):
    srv = hg.Server(max_slots=8, chunk_steps=7)
    try:
        jobs = []
        for i, (kw, nsteps, how) in enumerate(REQUESTS):
            p = params(hg, kw, how)
            st = None if how == "mode" else initial(hg, p, i)
            rid = srv.submit(p, nsteps, state=st, keep_state=True)
            jobs.append((rid, p, nsteps, st))
        for rid, p, nsteps, st in jobs:
            state = srv.wait(rid, timeout=300.0)
            if state == hg.model.REQ_FAILED:
                srv.result(rid)          # raises with the request's message
            assert state == hg.model.REQ_DONE
        stats = srv.stats()
        assert stats["completed"] == len(jobs)
        assert stats["max_holding"] >= 2          # requests overlapped on the device
        for rid, p, nsteps, st in jobs:
            info, fields = srv.result(rid)
            ref, step, t = alone(hg, p, nsteps, st)
            assert info["step"] == nsteps == step
            assert info["t"] == t
            assert info["t_submit"] <= info["t_admit"] <= info["t_start"] <= info["t_done"]
            for x, y in zip(fields, ref):
                if y is not None:
                    assert np.array_equal(x, y), "request %d differs from the model solved alone" % rid
    finally:
        srv.close()


def test_admission_follows_the_hbm_budget(hg):
    ps = [params(hg, REQUESTS[0][0], "mode"), params(hg, REQUESTS[3][0], "random"),
          params(hg, REQUESTS[0][0], "mode")]
    need = max(hg.footprint(p) for p in ps)
    srv = hg.Server(hbm_budget=1.05 * need, max_slots=8, chunk_steps=5)
    try:
        ids = [srv.submit(p, 10, state=None if p.ic == b"mode" else initial(hg, p, 9)) for p in ps]
        for rid in ids:
            assert srv.wait(rid, timeout=300.0) == hg.model.REQ_DONE
            info, _ = srv.result(rid)
            assert info["step"] == 10
        assert srv.stats()["max_holding"] == 1
        with pytest.raises(hg.HydftError):
            srv.submit(params(hg, dict(REQUESTS[3][0], nx=128, ny=128, nz=128), "mode"), 5)
    finally:
        srv.close()


def test_footprint_bounds_the_allocation(hg):
    for kw, _, how in REQUESTS:
        p = params(hg, kw, how)
        m = hg.Model(p)
        used = m.scalar("device_bytes")
        m.close()
        est = hg.footprint(p)
        assert used <= est <= 1.05 * used + 1e6


def test_failed_request_reports_its_error(hg):
    srv = hg.Server(max_slots=2)
    try:
        p = params(hg, REQUESTS[0][0], "random")
        n = np.full((p.nz, p.ny, p.nx), -1.0)
        rid = srv.submit(p, 5, state=(n, None, None))
        assert srv.wait(rid, timeout=120.0) == hg.model.REQ_FAILED
        with pytest.raises(hg.HydftError):
            srv.result(rid)
    finally:
        srv.close()


def test_results_collected_as_soon_as_requests_finish(hg):
    # a result may be collected before the server has released the request's
    # device memory; both orders must be safe
    srv = hg.Server(max_slots=4, chunk_steps=3)
    try:
        p = params(hg, REQUESTS[0][0], "mode")
        for k in range(6):
            rid = srv.submit(p, 2 + k % 3)
            assert srv.wait(rid, timeout=120.0) == hg.model.REQ_DONE
            info, _ = srv.result(rid)
            assert info["step"] == 2 + k % 3
        ids = [srv.submit(p, 3) for _ in range(4)]
        for rid in ids:
            srv.wait(rid, timeout=120.0)
            assert srv.result(rid)[0]["step"] == 3
    finally:
        srv.close()
