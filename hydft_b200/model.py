"""Python host over the C ABI of libhydft_gpu.so (include/hydft_gpu.h).

`Params` mirrors HyDFT's params_t (src/core/params.f90:17-78) and `Model`
mirrors model_t (src/model/model.f90:29-49): init, advance, rhs,
compute_dt, the public state n / mom / pi, t, dt and step, plus the spectral
probe (spec_t%mode) and the budgets of diag_t.  Every call runs the CUDA
path; there is no CPU fallback, and a missing library or GPU raises.

Fields use the reference's Fortran layout: a field n(nx,ny,nz) is a numpy
array of shape (nz, ny, nx); mom has shape (3, nz, ny, nx) and pi
(6, nz, ny, nx).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HYDFT_LIB") or os.path.join(_HERE, "lib", "libhydft_gpu.so")

_D, _I, _P = C.c_double, C.c_int, C.c_void_p

STATUS = {0: "OK", 1: "BAD_ARG", 2: "OOM", 3: "NONPOSITIVE_DENSITY", 4: "NONFINITE",
          5: "NEWTON", 6: "TIMEOUT", 7: "CUDA_ERROR", 8: "UNSUPPORTED", 9: "HNC", 10: "IO",
          11: "CFL"}


class HydftError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("hydft: %s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


class Params(C.Structure):
    """hydft_params: params_t as a POD struct (same names as the namelists)."""
    _fields_ = [
        ("nx", _I), ("ny", _I), ("nz", _I),
        ("lx", _D), ("ly", _D), ("lz", _D),
        ("dealias", _I),
        ("kind", C.c_char * 16),
        ("gamma", _D), ("kappa", _D), ("rs", _D), ("theta", _D), ("mass", _D),
        ("terms", C.c_char * 64),
        ("tfk_gamma", _D),
        ("closure", C.c_char * 16),
        ("transport", C.c_char * 16),
        ("eta", _D), ("xi", _D), ("tau", _D),
        ("tau_model", C.c_char * 16),
        ("adiabatic_index", _D),
        ("structure", C.c_char * 16),
        ("structure_file", C.c_char * 256),
        ("structure_kind", C.c_char * 4),
        ("hnc_nr", _I), ("hnc_maxiter", _I),
        ("hnc_rmax", _D), ("hnc_tol", _D), ("hnc_mix", _D),
        ("dt", _D), ("cfl", _D), ("tend", _D),
        ("nsteps_max", _I), ("iout", _I), ("iprobe", _I), ("idiag", _I),
        ("ic", C.c_char * 16),
        ("ic_amplitude", _D),
        ("ic_mode", _I * 3),
        ("ic_width", _D),
        ("ic_seed", _I),
        ("vext", C.c_char * 16),
        ("vext_amplitude", _D),
        ("vext_mode", _I * 3),
        ("vext_omega", _D), ("vext_width", _D), ("vext_ramp", _D),
        ("probe_mode", _I * 3),
        ("prefix", C.c_char * 256),
        ("gpu_precision", C.c_char * 8),
    ]


class Structure(C.Structure):
    _fields_ = [("n", _I), ("k", C.POINTER(_D)), ("c", C.POINTER(_D)),
                ("u_ex", _D), ("du_dgamma", _D), ("has_energy", _I)]


_lib = None


def lib():
    """Load libhydft_gpu.so (built by __graft_entry__.build())."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HydftError(7, "libhydft_gpu.so is not built (%s); run __graft_entry__.build()" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.hydft_params_default.argtypes = [C.POINTER(Params)]
        L.hydft_params_read.argtypes = [C.c_char_p, C.POINTER(Params)]
        L.hydft_params_finalize.argtypes = [C.POINTER(Params)]
        L.hydft_gpu_create.argtypes = [C.POINTER(Params), C.POINTER(Structure), _I, C.POINTER(_P)]
        L.hydft_gpu_destroy.argtypes = [_P]
        L.hydft_gpu_last_error.restype = C.c_char_p
        L.hydft_gpu_last_error.argtypes = [_P]
        L.hydft_gpu_create_error.restype = C.c_char_p
        L.hydft_gpu_set_state.argtypes = [_P, _P, _P, _P]
        L.hydft_gpu_get_state.argtypes = [_P, _P, _P, _P]
        L.hydft_gpu_set_initial_condition.argtypes = [_P, C.c_char_p, _D, C.POINTER(_I), _D, _I]
        L.hydft_gpu_advance.argtypes = [_P, _I]
        L.hydft_gpu_rhs.argtypes = [_P, _D, _P, _P, _P]
        L.hydft_gpu_compute_dt.argtypes = [_P, C.POINTER(_D)]
        L.hydft_gpu_get_time.argtypes = [_P, C.POINTER(_D), C.POINTER(_D), C.POINTER(C.c_int64)]
        L.hydft_gpu_set_time.argtypes = [_P, _D, _D]
        L.hydft_gpu_budgets.argtypes = [_P] + [C.POINTER(_D)] * 6
        L.hydft_gpu_mode.argtypes = [_P, _I, _I, _I, _I, C.POINTER(_D), C.POINTER(_D)]
        L.hydft_gpu_get_scalar.argtypes = [_P, C.c_char_p, C.POINTER(_D)]
        L.hydft_gpu_set_scalar.argtypes = [_P, C.c_char_p, _D]
        L.hydft_gpu_get_structure.argtypes = [_P, C.POINTER(_I), _P, _P]
        L.hydft_gpu_kernel.argtypes = [_P, _D, C.POINTER(_D)]
        L.hydft_gpu_profile.argtypes = [_P, _I, _I, C.c_char_p, _I, _P, _P, _P, C.POINTER(_I)]
        L.hydft_gpu_stream.restype = _P
        L.hydft_gpu_stream.argtypes = [_P]
        L.hydft_gpu_launch_count.restype = C.c_int64
        L.hydft_gpu_launch_count.argtypes = [_P]
        L.hydft_gpu_hnc_solve.argtypes = [C.c_char_p, _D, _D, _D, _D, _I, _D, _D, _D, _I, _I,
                                          _P, _P, _P, _P, _P, C.POINTER(_D), C.POINTER(_I),
                                          C.POINTER(_I), C.POINTER(_D)]
        L.hydft_gpu_fourier_bessel.argtypes = [_P, _P, _I, _D, _I, _I]
        L.hydft_gpu_fd_table.argtypes = [_I, _P, C.POINTER(_I)]
        L.hydft_gpu_fd_alpha.argtypes = [_I, _P, _P, _I]
        L.hydft_gpu_footprint.argtypes = [C.POINTER(Params), C.POINTER(_D)]
        L.hydft_gpu_write_fields.argtypes = [_P, C.c_char_p]
        L.hydft_gpu_read_fields.argtypes = [_P, C.c_char_p]
        L.hydft_gpu_run.argtypes = [_P]
        L.hydft_serve_create.argtypes = [_I, _D, _I, _I, C.POINTER(_P)]
        L.hydft_serve_submit.argtypes = [_P, C.POINTER(Params), _P, _P, _P, _I, _I, C.POINTER(C.c_int64)]
        L.hydft_serve_wait.argtypes = [_P, C.c_int64, _D, C.POINTER(_I)]
        L.hydft_serve_result.argtypes = [_P, C.c_int64, _P, _P, _P, _P]
        L.hydft_serve_stats.argtypes = [_P, _P]
        L.hydft_serve_destroy.argtypes = [_P]
        L.hydft_batch_create.argtypes = [_I, _P, _P, _I, C.POINTER(_P)]
        L.hydft_batch_destroy.argtypes = [_P]
        L.hydft_batch_size.argtypes = [_P]
        L.hydft_batch_member.argtypes = [_P, _I, C.POINTER(_P)]
        L.hydft_batch_advance.argtypes = [_P, _I]
        L.hydft_batch_last_error.restype = C.c_char_p
        L.hydft_batch_last_error.argtypes = [_P]
        L.hydft_batch_failed_member.argtypes = [_P]
        L.hydft_batch_launch_count.restype = C.c_int64
        L.hydft_batch_launch_count.argtypes = [_P]
        L.hydft_batch_stream.restype = _P
        L.hydft_batch_stream.argtypes = [_P]
        L.hydft_batch_grouped.argtypes = [_P, C.POINTER(_I), C.POINTER(_I)]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def default_params(**kw):
    """Params with the reference defaults and the given overrides."""
    p = Params()
    lib().hydft_params_default(C.byref(p))
    for k, v in kw.items():
        if k in ("ic_mode", "vext_mode", "probe_mode"):
            arr = getattr(p, k)
            for i in range(3):
                arr[i] = int(v[i])
        elif k == "dealias":
            p.dealias = 1 if v else 0
        elif isinstance(v, str):
            setattr(p, k, v.encode())
        else:
            setattr(p, k, v)
    return p


def read_params(path, base=None):
    """params_t%read of a namelist input file."""
    p = Params() if base is None else base
    if base is None:
        lib().hydft_params_default(C.byref(p))
    rc = lib().hydft_params_read(path.encode(), C.byref(p))
    if rc:
        raise HydftError(rc, lib().hydft_gpu_create_error().decode())
    return p


class Model:
    """model_t on the GPU."""

    def __init__(self, p, structure=None, device=0):
        L = lib()
        h = _P()
        st = None
        self._keep = None
        if structure is not None:
            k = np.ascontiguousarray(structure["k"], dtype=np.float64)
            c = np.ascontiguousarray(structure["c"], dtype=np.float64)
            self._keep = (k, c)
            st = Structure(k.size, k.ctypes.data_as(C.POINTER(_D)), c.ctypes.data_as(C.POINTER(_D)),
                           structure.get("u_ex", 0.0), structure.get("du_dgamma", 0.0),
                           1 if structure.get("has_energy", True) else 0)
        rc = L.hydft_gpu_create(C.byref(p), C.byref(st) if st is not None else None, device,
                                C.byref(h))
        if rc:
            raise HydftError(rc, L.hydft_gpu_create_error().decode())
        self.h = h
        self.p = p
        self.nx, self.ny, self.nz = p.nx, p.ny, p.nz
        self.shape = (p.nz, p.ny, p.nx)
        self.has_pi = bool(self.scalar("evolve"))

    @classmethod
    def _member(cls, h, p, owner):
        """A view of an ensemble member (the ensemble owns the handle)."""
        m = cls.__new__(cls)
        m._keep = None
        m.h = h
        m.p = p
        m._owner = owner
        m.nx, m.ny, m.nz = p.nx, p.ny, p.nz
        m.shape = (p.nz, p.ny, p.nx)
        m.has_pi = bool(m.scalar("evolve"))
        return m

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self.h = None
            return
        if getattr(self, "h", None):
            lib().hydft_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise HydftError(rc, lib().hydft_gpu_last_error(self.h).decode())

    # -- state
    def set_state(self, n, mom=None, pi=None):
        n = np.ascontiguousarray(n, dtype=np.float64).reshape(self.shape)
        mom = np.zeros((3,) + self.shape) if mom is None else np.ascontiguousarray(mom, dtype=np.float64)
        if self.has_pi:
            pi = np.zeros((6,) + self.shape) if pi is None else np.ascontiguousarray(pi, dtype=np.float64)
        else:
            pi = None
        self._check(lib().hydft_gpu_set_state(self.h, _ptr(n), _ptr(mom), _ptr(pi)))

    def get_state(self, out=None):
        """(n, mom, pi) as host arrays; `out` may supply the arrays to fill
        (C-contiguous float64, e.g. pinned buffers)."""
        if out is None:
            n = np.zeros(self.shape)
            mom = np.zeros((3,) + self.shape)
            pi = np.zeros((6,) + self.shape) if self.has_pi else None
        else:
            n, mom, pi = out
            if not self.has_pi:
                pi = None
        self._check(lib().hydft_gpu_get_state(self.h, _ptr(n), _ptr(mom), _ptr(pi)))
        return n, mom, pi

    @property
    def n(self):
        return self.get_state()[0]

    @property
    def mom(self):
        return self.get_state()[1]

    @property
    def pi(self):
        return self.get_state()[2]

    def set_initial_condition(self, kind, amplitude, mode=(1, 0, 0), width=1.0, seed=1234):
        md = (_I * 3)(*mode)
        self._check(lib().hydft_gpu_set_initial_condition(self.h, kind.encode(), amplitude, md,
                                                          width, seed))

    # -- files and the driver loop
    def write_fields(self, prefix):
        """write_fields: <prefix>_fld_NNNNNN.bin in the reference's format."""
        self._check(lib().hydft_gpu_write_fields(self.h, str(prefix).encode()))

    def read_fields(self, path):
        """Resume from a .bin field file (state, t; step from the name)."""
        self._check(lib().hydft_gpu_read_fields(self.h, str(path).encode()))

    def run(self):
        """hydft_run's loop from the current state, writing the prefix's
        _diag.dat, _probe.dat (and _fld_*.bin when iout > 0)."""
        self._check(lib().hydft_gpu_run(self.h))

    # -- stepping
    def advance(self, nsteps=1):
        self._check(lib().hydft_gpu_advance(self.h, int(nsteps)))

    def rhs(self, t):
        dn = np.zeros(self.shape)
        dmom = np.zeros((3,) + self.shape)
        dpi = np.zeros((6,) + self.shape) if self.has_pi else None
        self._check(lib().hydft_gpu_rhs(self.h, t, _ptr(dn), _ptr(dmom), _ptr(dpi)))
        return dn, dmom, dpi

    def compute_dt(self):
        dt = _D()
        self._check(lib().hydft_gpu_compute_dt(self.h, C.byref(dt)))
        return dt.value

    def _time(self):
        t, dt, st = _D(), _D(), C.c_int64()
        self._check(lib().hydft_gpu_get_time(self.h, C.byref(t), C.byref(dt), C.byref(st)))
        return t.value, dt.value, st.value

    @property
    def t(self):
        return self._time()[0]

    @property
    def dt(self):
        return self._time()[1]

    @dt.setter
    def dt(self, v):
        self._check(lib().hydft_gpu_set_time(self.h, self.t, float(v)))

    @property
    def step(self):
        return self._time()[2]

    def set_time(self, t, dt):
        self._check(lib().hydft_gpu_set_time(self.h, float(t), float(dt)))

    # -- diagnostics
    def budgets(self):
        mass, ek, fe, mn, mx = _D(), _D(), _D(), _D(), _D()
        mom = (_D * 3)()
        self._check(lib().hydft_gpu_budgets(self.h, C.byref(mass), mom, C.byref(ek), C.byref(fe),
                                            C.byref(mn), C.byref(mx)))
        return mass.value, np.array(list(mom)), ek.value, fe.value, mn.value, mx.value

    def mode(self, field, mx, my=0, mz=0):
        """Complex amplitude of mode (mx,my,mz) of n (field 0) or mom_i (1..3)."""
        re, im = _D(), _D()
        self._check(lib().hydft_gpu_mode(self.h, field, mx, my, mz, C.byref(re), C.byref(im)))
        return complex(re.value, im.value)

    def scalar(self, name):
        v = _D()
        self._check(lib().hydft_gpu_get_scalar(self.h, name.encode(), C.byref(v)))
        return v.value

    def set_scalar(self, name, value):
        self._check(lib().hydft_gpu_set_scalar(self.h, name.encode(), float(value)))

    def structure(self):
        n = _I()
        lib().hydft_gpu_get_structure(self.h, C.byref(n), None, None)
        k = np.zeros(n.value)
        c = np.zeros(n.value)
        lib().hydft_gpu_get_structure(self.h, C.byref(n), _ptr(k), _ptr(c))
        return k, c

    def kernel(self, k):
        v = _D()
        self._check(lib().hydft_gpu_kernel(self.h, float(k), C.byref(v)))
        return v.value

    def launch_count(self):
        return lib().hydft_gpu_launch_count(self.h)

    def stream_ptr(self):
        return lib().hydft_gpu_stream(self.h)

    def profile(self, nsteps=1):
        """Per-kernel CUDA-event timing of nsteps uncaptured steps:
        {name: (total_ms, bytes_per_launch, launches)}."""
        mk = 32
        names = C.create_string_buffer(1024)
        ms = np.zeros(mk)
        by = np.zeros(mk)
        nl = np.zeros(mk, dtype=np.int64)
        nk = _I()
        self._check(lib().hydft_gpu_profile(self.h, int(nsteps), mk, names, 1024, _ptr(ms), _ptr(by),
                                            _ptr(nl), C.byref(nk)))
        out = {}
        for i, nmx in enumerate(names.value.decode().split(",")[: nk.value]):
            out[nmx] = (float(ms[i]), float(by[i]), int(nl[i]))
        return out


def hnc_solve(potential, gamma, kappa, lam, n0, nr, rmax, tol, mix, maxiter, device=0):
    """OZ-HNC on the GPU (oz_hnc.f90:111-296); returns a dict of arrays."""
    out = {f: np.zeros(nr) for f in ("r", "k", "g", "ck", "sk")}
    u, conv, nit, res = _D(), _I(), _I(), _D()
    rc = lib().hydft_gpu_hnc_solve(potential.encode(), gamma, kappa, lam, n0, nr, rmax, tol, mix,
                                   maxiter, device, *(_ptr(out[f]) for f in ("r", "k", "g", "ck", "sk")),
                                   C.byref(u), C.byref(conv), C.byref(nit), C.byref(res))
    if rc:
        raise HydftError(rc, lib().hydft_gpu_create_error().decode())
    out.update(u_ex=u.value, converged=bool(conv.value), niter=nit.value, residual=res.value)
    return out


def fourier_bessel(f, rmax, direction, device=0):
    """fourier_bessel_t%r2k (direction 0) / %k2r (1) of a length-n array."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros_like(f)
    rc = lib().hydft_gpu_fourier_bessel(_ptr(f), _ptr(out), f.size, float(rmax), int(direction), device)
    if rc:
        raise HydftError(rc, lib().hydft_gpu_create_error().decode())
    return out


def fd_table(device=0):
    t = np.zeros(6 * 6601)
    n = _I()
    rc = lib().hydft_gpu_fd_table(device, _ptr(t), C.byref(n))
    if rc:
        raise HydftError(rc, lib().hydft_gpu_create_error().decode())
    return t.reshape(n.value, 6)


def fd_alpha(y, device=0):
    y = np.ascontiguousarray(y, dtype=np.float64)
    a = np.zeros_like(y)
    rc = lib().hydft_gpu_fd_alpha(device, _ptr(y), _ptr(a), y.size)
    if rc:
        raise HydftError(rc, lib().hydft_gpu_create_error().decode())
    return a


class Batch:
    """An ensemble of independent models advanced by one graph launch per
    step (hydft_batch_* in include/hydft_gpu.h).  `members[i]` is a Model
    view of member i for the single-model calls."""

    def __init__(self, params, structures=None, device=0):
        L = lib()
        n = len(params)
        arr = (Params * n)(*params)
        sts = None
        self._keep = []
        if structures is not None:
            sts = (Structure * n)()
            for i, st in enumerate(structures):
                if st is None:
                    sts[i].n = 0
                    continue
                k = np.ascontiguousarray(st["k"], dtype=np.float64)
                c = np.ascontiguousarray(st["c"], dtype=np.float64)
                self._keep.append((k, c))
                sts[i] = Structure(k.size, k.ctypes.data_as(C.POINTER(_D)), c.ctypes.data_as(C.POINTER(_D)),
                                   st.get("u_ex", 0.0), st.get("du_dgamma", 0.0),
                                   1 if st.get("has_energy", True) else 0)
        b = _P()
        rc = L.hydft_batch_create(n, C.cast(arr, _P), C.cast(sts, _P) if sts is not None else None, device,
                                  C.byref(b))
        if rc:
            raise HydftError(rc, L.hydft_gpu_create_error().decode())
        self.b = b
        self.params = list(params)
        self.members = []
        for i in range(n):
            h = _P()
            self._check(L.hydft_batch_member(b, i, C.byref(h)))
            self.members.append(Model._member(h, self.params[i], self))

    def _check(self, rc):
        if rc:
            raise HydftError(rc, lib().hydft_batch_last_error(self.b).decode())

    def __len__(self):
        return len(self.members)

    def advance(self, nsteps=1):
        self._check(lib().hydft_batch_advance(self.b, int(nsteps)))

    def failed_member(self):
        return lib().hydft_batch_failed_member(self.b)

    def grouped(self):
        """(groups, members in groups) of the last captured ensemble step:
        members in a group share every launch of the step."""
        g, m = _I(), _I()
        lib().hydft_batch_grouped(self.b, C.byref(g), C.byref(m))
        return g.value, m.value

    def launch_count(self):
        return lib().hydft_batch_launch_count(self.b)

    def stream_ptr(self):
        return lib().hydft_batch_stream(self.b)

    def close(self):
        if getattr(self, "b", None):
            for m in self.members:
                m.h = None
            lib().hydft_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(p):
    """Device bytes a model of params p allocates (hydft_gpu_footprint)."""
    b = _D()
    rc = lib().hydft_gpu_footprint(C.byref(p), C.byref(b))
    if rc:
        raise HydftError(rc, "invalid grid")
    return b.value


REQ_QUEUED, REQ_SETUP, REQ_RUNNING, REQ_DONE, REQ_FAILED = range(5)
INFO_KEYS = ("t", "dt", "step", "mass", "mom_x", "mom_y", "mom_z", "ekin", "nmin", "nmax",
             "t_submit", "t_admit", "t_start", "t_done", "bytes", "launches")


class Server:
    """Continuous-batching solve server on one GPU (hydft_serve_*)."""

    def __init__(self, device=0, hbm_budget=0.0, max_slots=64, chunk_steps=50):
        b = _P()
        rc = lib().hydft_serve_create(device, float(hbm_budget), max_slots, chunk_steps, C.byref(b))
        if rc:
            raise HydftError(rc, lib().hydft_gpu_create_error().decode())
        self.s = b
        self._shapes = {}

    def submit(self, p, nsteps, state=None, keep_state=False):
        """Queue a solve of params p for nsteps steps; state = (n, mom, pi)
        host arrays or None for p's initial condition.  Returns its id."""
        rid = C.c_int64()
        keep = []
        ptrs = [None, None, None]
        if state is not None:
            shp = (p.nz, p.ny, p.nx)
            n = np.ascontiguousarray(state[0], dtype=np.float64).reshape(shp)
            mom = np.zeros((3,) + shp) if state[1] is None else np.ascontiguousarray(state[1], dtype=np.float64)
            pi = None if len(state) < 3 or state[2] is None else np.ascontiguousarray(state[2], dtype=np.float64)
            keep = [n, mom, pi]
            ptrs = [_ptr(n), _ptr(mom), _ptr(pi)]
        rc = lib().hydft_serve_submit(self.s, C.byref(p), ptrs[0], ptrs[1], ptrs[2], int(nsteps),
                                      1 if keep_state else 0, C.byref(rid))
        if rc:
            raise HydftError(rc, lib().hydft_gpu_create_error().decode())
        self._shapes[rid.value] = ((p.nz, p.ny, p.nx), p.closure.decode() == "maxwell", keep_state)
        return rid.value

    def wait(self, rid, timeout=-1.0):
        st = _I()
        rc = lib().hydft_serve_wait(self.s, rid, float(timeout), C.byref(st))
        if rc:
            raise HydftError(rc, "unknown request %d" % rid)
        return st.value

    def result(self, rid):
        """Final scalars (dict) and, if kept, fields (n, mom, pi) of a finished
        request; raises HydftError if it failed.  Releases the request."""
        shp, maxwell, keep = self._shapes.pop(rid)
        info = np.zeros(16)
        n = mom = pi = None
        if keep:
            n = np.zeros(shp)
            mom = np.zeros((3,) + shp)
            pi = np.zeros((6,) + shp) if maxwell else None
        rc = lib().hydft_serve_result(self.s, rid, _ptr(n), _ptr(mom), _ptr(pi), _ptr(info))
        if rc:
            raise HydftError(rc, lib().hydft_gpu_create_error().decode())
        return dict(zip(INFO_KEYS, info.tolist())), (n, mom, pi)

    def stats(self):
        v = np.zeros(6)
        lib().hydft_serve_stats(self.s, _ptr(v))
        return dict(zip(("queued", "holding", "completed", "max_holding", "bytes_in_use", "budget"), v.tolist()))

    def close(self):
        if getattr(self, "s", None):
            lib().hydft_serve_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
