"""ctypes access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C FP64 restatement of the HyDFT solver step (see
oracle/oracle.h).  Only the tests, the smoke check and the CPU-baseline leg of
the benchmark use this module, and only as the reference the device results
are compared with.

Arrays follow the reference's Fortran layout: a field u(nx,ny,nz) is a numpy
array of shape (nz, ny, nx) in C order; a half spectrum has shape
(nz, ny, nx//2+1); a vector field has a leading component axis.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

TERMS = {"ideal": 1, "tf": 2, "gradient": 3, "hartree": 4, "ry": 5}
VEXT = {"none": 0, "mode": 1, "driven": 2, "gaussian": 3}
TRANSPORT = {"constant": 0, "yukawa_fit": 1, "stanton_murillo": 2, "electron_fit": 3}
POT = {"yukawa": 0, "coulomb": 1, "hansen_mcdonald": 2, "hm": 2, "qsp": 2}

_D = C.c_double
_I = C.c_int
_P = C.c_void_p
_DP = C.POINTER(C.c_double)


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", _I), ("ny", _I), ("nz", _I),
        ("lx", _D), ("ly", _D), ("lz", _D),
        ("dealias", _I), ("electron", _I),
        ("gamma", _D), ("kappa", _D), ("rs", _D), ("theta", _D), ("mass", _D),
        ("nterms", _I), ("terms", _I * 8),
        ("tfk_gamma", _D),
        ("maxwell", _I), ("transport", _I),
        ("eta", _D), ("xi", _D), ("tau", _D),
        ("tau_ichimaru", _I),
        ("adiabatic_index", _D),
        ("hnc_nr", _I), ("hnc_maxiter", _I),
        ("hnc_rmax", _D), ("hnc_tol", _D), ("hnc_mix", _D),
        ("dt", _D), ("cfl", _D),
        ("vext", _I),
        ("vext_amplitude", _D), ("vext_omega", _D), ("vext_width", _D), ("vext_ramp", _D),
        ("vext_mode", _I * 3),
    ]


class OrcPot(C.Structure):
    _fields_ = [("kind", _I), ("gamma", _D), ("kappa", _D), ("ksplit", _D),
                ("lam", _D), ("pauli", _I)]


class OrcStructure(C.Structure):
    _fields_ = [("n", _I), ("n0", _D), ("k", _DP), ("c", _DP), ("s", _DP),
                ("u_ex", _D), ("du_dgamma", _D), ("has_energy", _I)]


class _Cplx(C.Structure):
    _fields_ = [("re", _D), ("im", _D)]


class OrcHncResult(C.Structure):
    _fields_ = [("nr", _I), ("n0", _D), ("dr", _D), ("dk", _D),
                ("r", _DP), ("k", _DP), ("g", _DP), ("cr", _DP), ("ck", _DP),
                ("hk", _DP), ("sk", _DP), ("u_ex", _D), ("converged", _I),
                ("niter", _I), ("residual", _D)]


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_params_default.argtypes = [C.POINTER(OrcParams)]
        L.orc_model_create.restype = _P
        L.orc_model_create.argtypes = [C.POINTER(OrcParams), _P, C.POINTER(_I)]
        L.orc_model_destroy.argtypes = [_P]
        for name in ("orc_model_n", "orc_model_mom", "orc_model_pi", "orc_model_mu",
                     "orc_model_vext_v"):
            getattr(L, name).restype = _DP
            getattr(L, name).argtypes = [_P]
        L.orc_model_get.restype = _D
        L.orc_model_get.argtypes = [_P, C.c_char_p]
        L.orc_model_set.argtypes = [_P, C.c_char_p, _D]
        L.orc_model_rhs.argtypes = [_P, _D, _P, _P, _P]
        L.orc_model_advance.argtypes = [_P]
        L.orc_model_stage.argtypes = [_P, _I]
        L.orc_model_compute_dt.argtypes = [_P]
        L.orc_model_ncells.argtypes = [_P]
        L.orc_model_has_pi.argtypes = [_P]
        L.orc_model_fft_count.restype = C.c_long
        L.orc_model_fft_count.argtypes = [_P]
        L.orc_model_set_ic.argtypes = [_P, _I, _D, C.POINTER(_I), _D]
        L.orc_model_budgets.argtypes = [_P, _DP, _DP, _DP, _DP]
        L.orc_model_nterms.argtypes = [_P]
        L.orc_model_term_id.argtypes = [_P, _I]
        L.orc_model_term_add_mu.argtypes = [_P, _I, _P, _P, _P]
        L.orc_model_term_kernel.restype = _D
        L.orc_model_term_kernel.argtypes = [_P, _I, _D]
        L.orc_model_kernel.restype = _D
        L.orc_model_kernel.argtypes = [_P, _D]
        L.orc_model_mu_total.argtypes = [_P, _P, _P, _P]
        L.orc_model_energy.restype = _D
        L.orc_model_energy.argtypes = [_P, _P, _P]
        L.orc_model_spec.restype = _P
        L.orc_model_spec.argtypes = [_P]
        L.orc_spec_fwd.argtypes = [_P, _P, _P]
        L.orc_spec_bwd.argtypes = [_P, _P, _P]
        L.orc_linear_c2.restype = _D
        L.orc_linear_c2.argtypes = [_P, _D]
        L.orc_linear_chi.restype = _Cplx
        L.orc_linear_chi.argtypes = [_P, _D, _D]
        L.orc_linear_dispersion.restype = _Cplx
        L.orc_linear_dispersion.argtypes = [_P, _D]
        L.orc_linear_dsf.restype = _D
        L.orc_linear_dsf.argtypes = [_P, _D, _D]
        L.orc_fit_damped_mode.argtypes = [_I, _P, _P, _D, _DP, _DP, C.POINTER(_I)]
        L.orc_fit_driven_response.argtypes = [_I, _P, _P, _D, _D, _P, _DP]
        for name in ("orc_fd_im12", "orc_fd_ip12", "orc_fd_ip32", "orc_fd_dim12",
                     "orc_fd_d2im12", "orc_fd_xi", "orc_fd_dxi"):
            getattr(L, name).restype = _D
            getattr(L, name).argtypes = [_D]
        L.orc_fd_alpha_from_ip12.restype = _D
        L.orc_fd_alpha_from_ip12.argtypes = [_D, C.POINTER(_I)]
        L.orc_fd_table.restype = _DP
        L.orc_fd_table.argtypes = [C.POINTER(_I)]
        L.orc_fft1_c.argtypes = [_I, _P, _I]
        L.orc_fft3_create.restype = _P
        L.orc_fft3_create.argtypes = [_I, _I, _I]
        L.orc_fft3_destroy.argtypes = [_P]
        L.orc_fft3_fwd.argtypes = [_P, _P, _P]
        L.orc_fft3_bwd.argtypes = [_P, _P, _P]
        L.orc_dst1_create.restype = _P
        L.orc_dst1_create.argtypes = [_I]
        L.orc_dst1_destroy.argtypes = [_P]
        L.orc_dst1_exec.argtypes = [_P, _P, _P]
        L.orc_fb_r2k.argtypes = [_I, _D, _P, _P]
        L.orc_fb_k2r.argtypes = [_I, _D, _P, _P]
        L.orc_hnc_solve.argtypes = [C.POINTER(OrcPot), _D, _I, _D, _D, _D, _I,
                                    C.POINTER(OrcHncResult)]
        L.orc_hnc_result_free.argtypes = [C.POINTER(OrcHncResult)]
        L.orc_structure_from_hnc.argtypes = [C.POINTER(OrcPot), _D, _I, _D, _D, _D, _I, _I,
                                             C.POINTER(OrcStructure)]
        L.orc_structure_free.argtypes = [C.POINTER(OrcStructure)]
        L.orc_structure_set.argtypes = [C.POINTER(OrcStructure), _I, _P, _P, _D, _D, _D, _I]
        L.orc_structure_c_of_k.restype = _D
        L.orc_structure_c_of_k.argtypes = [C.POINTER(OrcStructure), _D]
        L.orc_sm_knm.restype = _D
        L.orc_sm_knm.argtypes = [_I, _D]
        L.orc_sm_viscosity.restype = _D
        L.orc_sm_viscosity.argtypes = [_D, _D]
        L.orc_sm_diffusion.restype = _D
        L.orc_sm_diffusion.argtypes = [_D, _D]
        L.orc_sm_conductivity.restype = _D
        L.orc_sm_conductivity.argtypes = [_D, _D]
        L.orc_sm_electron_viscosity.argtypes = [_D, _D, _D, _D, _DP, _DP, _DP]
        L.orc_set_threads.argtypes = [_I]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def set_threads(n):
    lib().orc_set_threads(int(n))


# ----------------------------------------------------------------- FFT
def fft1(x, sign=-1):
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().orc_fft1_c(a.size, _ptr(a), sign)
    return a


class FFT3:
    def __init__(self, nx, ny, nz):
        self.shape = (nz, ny, nx)
        self.hshape = (nz, ny, nx // 2 + 1)
        self.h = lib().orc_fft3_create(nx, ny, nz)

    def fwd(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.shape)
        out = np.zeros(self.hshape, dtype=np.complex128)
        lib().orc_fft3_fwd(self.h, _ptr(u), _ptr(out))
        return out

    def bwd(self, uh):
        uh = np.ascontiguousarray(uh, dtype=np.complex128).reshape(self.hshape)
        out = np.zeros(self.shape)
        lib().orc_fft3_bwd(self.h, _ptr(uh), _ptr(out))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_fft3_destroy(self.h)
            self.h = None


def dst1(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    d = lib().orc_dst1_create(x.size)
    lib().orc_dst1_exec(d, _ptr(x), _ptr(y))
    lib().orc_dst1_destroy(d)
    return y


def fb_r2k(fr, rmax):
    fr = np.ascontiguousarray(fr, dtype=np.float64)
    fk = np.zeros_like(fr)
    lib().orc_fb_r2k(fr.size, rmax, _ptr(fr), _ptr(fk))
    return fk


def fb_k2r(fk, rmax):
    fk = np.ascontiguousarray(fk, dtype=np.float64)
    fr = np.zeros_like(fk)
    lib().orc_fb_k2r(fk.size, rmax, _ptr(fk), _ptr(fr))
    return fr


# ----------------------------------------------------------- special
def fd(name, a):
    return getattr(lib(), "orc_fd_" + name)(float(a))


def fd_alpha_from_ip12(y):
    st = _I(0)
    v = lib().orc_fd_alpha_from_ip12(float(y), C.byref(st))
    return v, st.value


def fd_table():
    n = _I(0)
    p = lib().orc_fd_table(C.byref(n))
    return np.ctypeslib.as_array(p, shape=(n.value, 6)).copy()


# --------------------------------------------------------------- HNC
class HncResult:
    pass


def make_pot(name, gamma, kappa=0.0, lam=1.0, pauli=True):
    return OrcPot(POT[name.lower()], gamma, kappa, 1.0, lam, 1 if pauli else 0)


def hnc_solve(pot, n0, nr, rmax, tol, mix, maxiter):
    res = OrcHncResult()
    rc = lib().orc_hnc_solve(C.byref(pot), n0, nr, rmax, tol, mix, maxiter, C.byref(res))
    out = HncResult()
    out.rc = rc
    out.converged = bool(res.converged)
    out.niter = res.niter
    out.residual = res.residual
    out.u_ex = res.u_ex
    if res.r:
        n = res.nr
        for f in ("r", "k", "g", "cr", "ck", "hk", "sk"):
            setattr(out, f, np.ctypeslib.as_array(getattr(res, f), shape=(n,)).copy())
    lib().orc_hnc_result_free(C.byref(res))
    return out


class Structure:
    """structure_t from the HNC source (structure_source.f90:50-83)."""

    def __init__(self, k, c, n0, u_ex=0.0, du_dgamma=0.0, has_energy=True):
        self.k = np.ascontiguousarray(k, dtype=np.float64)
        self.c = np.ascontiguousarray(c, dtype=np.float64)
        self.n0 = n0
        self.u_ex = u_ex
        self.du_dgamma = du_dgamma
        self.has_energy = has_energy

    def c_struct(self):
        st = OrcStructure()
        lib().orc_structure_set(C.byref(st), self.k.size, _ptr(self.k), _ptr(self.c), self.n0,
                                self.u_ex, self.du_dgamma, 1 if self.has_energy else 0)
        return st

    def c_of_k(self, q):
        st = self.c_struct()
        v = lib().orc_structure_c_of_k(C.byref(st), q)
        lib().orc_structure_free(C.byref(st))
        return v

    def s_of_k(self, q):
        return 1.0 / (1.0 - self.n0 * self.c_of_k(q))


def structure_from_hnc(pot, n0, nr, rmax, tol, mix, maxiter, with_derivative=False):
    st = OrcStructure()
    rc = lib().orc_structure_from_hnc(C.byref(pot), n0, nr, rmax, tol, mix, maxiter,
                                      1 if with_derivative else 0, C.byref(st))
    if rc:
        raise RuntimeError("structure_from_hnc failed (%d)" % rc)
    n = st.n
    out = Structure(np.ctypeslib.as_array(st.k, shape=(n,)).copy(),
                    np.ctypeslib.as_array(st.c, shape=(n,)).copy(), st.n0, st.u_ex,
                    st.du_dgamma, bool(st.has_energy))
    lib().orc_structure_free(C.byref(st))
    return out


def structure_from_file(path, kind, n0):
    """structure_from_file (structure_source.f90:87-138): a two-column text
    file (k, S(k)) for kind 's' or (k, c(k)) for kind 'c'; blank lines,
    lines starting with '#' and lines whose first two entries are not
    numbers are skipped; k must be positive and strictly increasing."""
    kk, vv = [], []
    with open(path) as f:
        for line in f:
            t = line.strip()
            if not t or t.startswith("#"):
                continue
            parts = t.replace(",", " ").split()
            try:
                a = float(parts[0].replace("d", "e").replace("D", "e"))
                b = float(parts[1].replace("d", "e").replace("D", "e"))
            except (ValueError, IndexError):
                continue
            kk.append(a)
            vv.append(b)
    if len(kk) < 2:
        raise ValueError("structure file has fewer than two data rows: " + path)
    k = np.array(kk)
    v = np.array(vv)
    kind = kind[:1].lower()
    if kind == "s":
        c = (1.0 - 1.0 / v) / n0
    elif kind == "c":
        c = v
    else:
        raise ValueError("structure file kind must be s or c")
    if np.any(k[1:] <= k[:-1]):
        raise ValueError("structure file: k must be strictly increasing")
    if k[0] <= 0.0:
        raise ValueError("structure file: k must be positive")
    return Structure(k, c, n0, 0.0, 0.0, False)


# transport fits (stanton_murillo.f90)
def sm_knm(idx, g):
    return lib().orc_sm_knm(idx, g)


def sm_viscosity(gamma, kappa):
    return lib().orc_sm_viscosity(gamma, kappa)


def sm_diffusion(gamma, kappa):
    return lib().orc_sm_diffusion(gamma, kappa)


def sm_conductivity(gamma, kappa):
    return lib().orc_sm_conductivity(gamma, kappa)


def sm_electron_viscosity(rs, gamma, theta, lambda_tf):
    el, cv, sm = _D(), _D(), _D()
    lib().orc_sm_electron_viscosity(rs, gamma, theta, lambda_tf, C.byref(el), C.byref(cv), C.byref(sm))
    return el.value, cv.value, sm.value


# ------------------------------------------------------------- params
def params(**kw):
    """An orc_params with the reference defaults (params.f90:17-78) and the
    given overrides, using the reference's names and string values."""
    p = OrcParams()
    lib().orc_params_default(C.byref(p))
    for key, val in kw.items():
        if key == "kind":
            p.electron = 1 if val == "electron" else 0
        elif key == "terms":
            names = [t.strip() for t in val.split(",") if t.strip()] if val else []
            p.nterms = len(names)
            for i, t in enumerate(names):
                p.terms[i] = TERMS[t]
        elif key == "closure":
            p.maxwell = 1 if val == "maxwell" else 0
        elif key == "transport":
            p.transport = TRANSPORT[val]
        elif key == "tau_model":
            p.tau_ichimaru = 1 if val == "ichimaru" else 0
        elif key == "vext":
            p.vext = VEXT[val]
        elif key == "vext_mode":
            for i in range(3):
                p.vext_mode[i] = int(val[i])
        elif key == "dealias":
            p.dealias = 1 if val else 0
        else:
            setattr(p, key, val)
    return p


class Model:
    """model_t (model.f90:29-49) on the CPU."""

    def __init__(self, p, structure=None):
        self.p = p
        L = lib()
        st_c = structure.c_struct() if structure is not None else None
        status = _I(0)
        self.h = L.orc_model_create(C.byref(p), C.byref(st_c) if st_c is not None else None,
                                    C.byref(status))
        if st_c is not None:
            L.orc_structure_free(C.byref(st_c))
        if not self.h:
            raise RuntimeError("oracle model_create failed (status %d)" % status.value)
        self.nx, self.ny, self.nz = p.nx, p.ny, p.nz
        self.shape = (p.nz, p.ny, p.nx)
        self.hshape = (p.nz, p.ny, p.nx // 2 + 1)
        self.nc = p.nx * p.ny * p.nz
        self.has_pi = bool(L.orc_model_has_pi(self.h))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_model_destroy(self.h)
            self.h = None

    # state views (live)
    def _view(self, fn, ncomp):
        p = fn(self.h)
        if not p:
            return None
        shp = self.shape if ncomp == 1 else (ncomp,) + self.shape
        return np.ctypeslib.as_array(p, shape=shp)

    @property
    def n(self):
        return self._view(lib().orc_model_n, 1)

    @property
    def mom(self):
        return self._view(lib().orc_model_mom, 3)

    @property
    def pi(self):
        return self._view(lib().orc_model_pi, 6) if self.has_pi else None

    @property
    def mu(self):
        return self._view(lib().orc_model_mu, 1)

    @property
    def vext_v(self):
        return self._view(lib().orc_model_vext_v, 1)

    def get(self, name):
        return lib().orc_model_get(self.h, name.encode())

    def set(self, name, v):
        lib().orc_model_set(self.h, name.encode(), float(v))

    @property
    def t(self):
        return self.get("t")

    @property
    def dt(self):
        return self.get("dt")

    @property
    def step(self):
        return int(self.get("step"))

    def set_state(self, n, mom=None, pi=None):
        self.n[...] = n
        self.mom[...] = 0.0 if mom is None else mom
        if self.has_pi:
            self.pi[...] = 0.0 if pi is None else pi

    def set_ic(self, kind, amp, mode=(1, 0, 0), width=1.0):
        k = {"uniform": 0, "mode": 1, "random": 2, "gaussian": 3}[kind]
        md = (_I * 3)(*mode)
        rc = lib().orc_model_set_ic(self.h, k, amp, md, width)
        if rc:
            raise RuntimeError("set_initial_condition failed (%d)" % rc)

    def rhs(self, t):
        dn = np.zeros(self.shape)
        dmom = np.zeros((3,) + self.shape)
        dpi = np.zeros((6,) + self.shape)
        rc = lib().orc_model_rhs(self.h, t, _ptr(dn), _ptr(dmom), _ptr(dpi))
        if rc:
            raise RuntimeError("rhs failed (%d)" % rc)
        return dn, dmom, dpi

    def compute_dt(self):
        rc = lib().orc_model_compute_dt(self.h)
        if rc:
            raise RuntimeError("compute_dt failed (%d)" % rc)
        return self.dt

    def advance(self, nsteps=1):
        for _ in range(nsteps):
            rc = lib().orc_model_advance(self.h)
            if rc:
                raise RuntimeError("advance failed (%d)" % rc)

    def stage(self, s):
        """Stage s (0, 1, 2) of one RK3 step alone; stages 0, 1, 2 in order
        are one advance()."""
        rc = lib().orc_model_stage(self.h, int(s))
        if rc:
            raise RuntimeError("stage failed (%d)" % rc)

    def fft_count(self):
        return lib().orc_model_fft_count(self.h)

    def fwd(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(self.hshape, dtype=np.complex128)
        lib().orc_spec_fwd(lib().orc_model_spec(self.h), _ptr(u), _ptr(out))
        return out

    def mode(self, u, mx, my, mz):
        uh = self.fwd(u)
        return uh[mz % self.nz, my % self.ny, mx]

    def budgets(self):
        mass, ek, fe = _D(), _D(), _D()
        mom = (_D * 3)()
        lib().orc_model_budgets(self.h, C.byref(mass), mom, C.byref(ek), C.byref(fe))
        return mass.value, np.array(list(mom)), ek.value, fe.value

    def nterms(self):
        return lib().orc_model_nterms(self.h)

    def term_name(self, i):
        tid = lib().orc_model_term_id(self.h, i)
        return {v: k for k, v in TERMS.items()}[tid]

    def term_add_mu(self, i, n, nhat, mu):
        n = np.ascontiguousarray(n, dtype=np.float64)
        nhat = np.ascontiguousarray(nhat, dtype=np.complex128)
        rc = lib().orc_model_term_add_mu(self.h, i, _ptr(n), _ptr(nhat), _ptr(mu))
        if rc:
            raise RuntimeError("add_mu failed (%d)" % rc)

    def term_kernel(self, i, k):
        return lib().orc_model_term_kernel(self.h, i, k)

    def kernel(self, k):
        return lib().orc_model_kernel(self.h, k)

    def mu_total(self, n, nhat):
        n = np.ascontiguousarray(n, dtype=np.float64)
        nhat = np.ascontiguousarray(nhat, dtype=np.complex128)
        mu = np.zeros(self.shape)
        rc = lib().orc_model_mu_total(self.h, _ptr(n), _ptr(nhat), _ptr(mu))
        if rc:
            raise RuntimeError("mu failed (%d)" % rc)
        return mu

    # linear response
    def c2(self, k):
        return lib().orc_linear_c2(self.h, k)

    def chi(self, k, w):
        r = lib().orc_linear_chi(self.h, k, w)
        return complex(r.re, r.im)

    def dispersion(self, k):
        r = lib().orc_linear_dispersion(self.h, k)
        return complex(r.re, r.im)

    def dsf(self, k, w):
        return lib().orc_linear_dsf(self.h, k, w)


def fit_damped_mode(t, y, t_start):
    t = np.ascontiguousarray(t, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    om, ga, nz = _D(), _D(), _I()
    lib().orc_fit_damped_mode(t.size, _ptr(t), _ptr(y), t_start, C.byref(om), C.byref(ga),
                              C.byref(nz))
    return om.value, ga.value, nz.value


def fit_driven_response(t, z, w, t_start):
    t = np.ascontiguousarray(t, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.complex128)
    a = np.zeros(1, dtype=np.complex128)
    sc = _D()
    lib().orc_fit_driven_response(t.size, _ptr(t), _ptr(z), w, t_start, _ptr(a), C.byref(sc))
    return complex(a[0]), sc.value
