"""The C-ABI library: it loads, exports every entry point declared in
include/hydft_gpu.h, and its host-only parts (namelist input, defaults)
behave like params_t.  No GPU is needed; on a machine without one,
hydft_gpu_create must fail loudly (there is no CPU path)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "hydft_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hydft_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import hydft_b200
    L = hydft_b200.lib()
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_params_defaults():
    import hydft_b200 as hg
    p = hg.default_params()
    # params.f90:17-78
    assert (p.nx, p.ny, p.nz) == (64, 1, 1)
    assert p.lx == 20.0 and p.dealias == 1
    assert p.kind == b"ion" and p.closure == b"newtonian" and p.transport == b"constant"
    assert p.hnc_nr == 8192 and p.hnc_rmax == 80.0 and p.hnc_tol == 1e-9 and p.hnc_mix == 0.2
    assert p.cfl == 0.4 and p.iprobe == 1 and p.idiag == 10
    assert abs(p.tfk_gamma - 1.0 / 9.0) < 1e-16
    assert p.gpu_precision == b"fp64"


def test_params_read_namelist(tmp_path):
    import hydft_b200 as hg
    f = tmp_path / "hydft.in"
    f.write_text("""! a HyDFT input deck
&grid nx=32 ny=16, nz=8 lx=20.0 ly=10.D0 lz=5 dealias=.false. /
&species kind='Electron' rs=1.0 theta=1.0 closure='maxwell'
         transport='electron_fit' tau_model='constant' tau=2.5 /
&time dt=0.01 cfl=0.3 /
&external type='driven' amplitude=1e-4 mode=3,0,0 omega=0.7 ramp=10 /
&gpu precision='fp32' /
""")
    p = hg.read_params(str(f))
    assert (p.nx, p.ny, p.nz) == (32, 16, 8)
    assert p.ly == 10.0 and p.lz == 5.0 and p.dealias == 0
    assert p.kind == b"electron"
    # derived defaults (params.f90:161-172)
    assert p.terms == b"tf,gradient,hartree,ry"
    import math
    assert abs(p.gamma - 2.0 * 1.0 / (1.0 * (9 * math.pi / 4) ** (2.0 / 3.0))) < 1e-15
    assert p.kappa == 0.0
    assert p.closure == b"maxwell" and p.tau == 2.5 and p.tau_model == b"constant"
    assert p.vext == b"driven" and list(p.vext_mode) == [3, 0, 0] and p.vext_omega == 0.7
    assert p.dt == 0.01 and p.cfl == 0.3
    assert p.gpu_precision == b"fp32"


def test_params_read_errors(tmp_path):
    import hydft_b200 as hg
    with pytest.raises(hg.HydftError):
        hg.read_params(str(tmp_path / "missing.in"))
    f = tmp_path / "bad.in"
    f.write_text("&grid nx=abc /\n")
    with pytest.raises(hg.HydftError):
        hg.read_params(str(f))


def test_create_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import hydft_b200 as hg
    with pytest.raises(hg.HydftError) as e:
        hg.Model(hg.default_params(nx=16))
    assert e.value.code == 7


def test_footprint_of_the_256_maxwell_step():
    import hydft_b200 as hg
    kw = dict(kind="ion", nx=256, ny=256, nz=256, lx=64.0, ly=64.0, lz=64.0, closure="maxwell")
    f32 = hg.footprint(hg.default_params(gpu_precision="fp32", **kw))
    f64 = hg.footprint(hg.default_params(gpu_precision="fp64", **kw))
    newt = hg.footprint(hg.default_params(gpu_precision="fp32", **dict(kw, closure="newtonian")))
    assert 3.5e9 < f32 < 5.0e9
    assert 1.9 < f64 / f32 < 2.0      # everything doubles but the FP64 staging field
    assert newt < f32
