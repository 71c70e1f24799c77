"""impact_b200 -- Python host side of the B200 implementation of IMPACT's fractional-step hot path.

Everything here is a thin ctypes layer over ``libimpact_b200.so`` (the CUDA kernels and the C
ABI declared in ``include/impact_b200.h``).  There is no CPU fallback: if the shared library is
missing or cannot be loaded, every entry point raises.

* ``Grid``       -- coordinates and FD coefficient tables of one periodic grid (FD_coeffs,
                    mod_coeffs.f90:37-112; get_stencil, mod_coeffs.f90:1048).
* ``Case``       -- one vessel case resident on one GPU: fields, Poisson solve, RK3 steps.
* ``launchers``  -- the reference's launcher FFI (``gradient_launcher_`` ...) on device pointers.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libimpact_b200.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_uint8)
_vp = C.c_void_p

FIELDS = {"vel1": 0, "vel2": 1, "vel3": 2, "pre": 3, "nl1": 4, "nl2": 5, "nl3": 6, "res": 7,
          "rhs1": 8, "rhs2": 9, "rhs3": 10}


class ImpactError(RuntimeError):
    pass


class AxisTables(C.Structure):
    _fields_ = [(n, _dp) for n in ("cG", "cD", "cIpu", "cIup", "cNpU", "cNpD", "cNuU", "cNuD",
                                   "cp1", "cpp", "cuu", "cdg")]


class Coeffs(C.Structure):
    _fields_ = [("axis", C.POINTER(AxisTables) * 3), ("xp", _dp * 3), ("xu", _dp * 3), ("L", C.c_double * 3)]


class CaseDesc(C.Structure):
    _fields_ = [("N1", C.c_int), ("N2", C.c_int), ("N3", C.c_int), ("precision", C.c_int),
                ("device", C.c_int), ("stream", _vp)]


class SolverParams(C.Structure):
    _fields_ = [("tol_rel", C.c_double), ("tol_abs_inf", C.c_double), ("max_it", C.c_int),
                ("n_sweeps", C.c_int), ("omega", C.c_double), ("init_yes", C.c_int),
                ("check_every", C.c_int), ("inner_tol_rel", C.c_double), ("inner_max_it", C.c_int),
                ("precond", C.c_int), ("mg_down", C.c_int), ("mg_up", C.c_int), ("mg_bottom", C.c_int),
                ("tile_kc", C.c_int), ("smooth_unfused", C.c_int), ("bottom_cheb", C.c_int)]


class SolverResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("inner_iterations", C.c_int), ("status", C.c_int),
                ("res_inf", C.c_double), ("res_two", C.c_double), ("b_two", C.c_double)]


class StepParams(C.Structure):
    _fields_ = [("Re", C.c_double), ("CFL", C.c_double), ("dtime_max", C.c_double),
                ("dtime0", C.c_double), ("U0", C.c_double), ("T_pulse", C.c_double),
                ("level_pressure", C.c_int), ("poisson", SolverParams), ("explicit_fp32", C.c_int)]


class StepState(C.Structure):
    _fields_ = [("time", C.c_double), ("dtime", C.c_double), ("timestep", C.c_int),
                ("poisson_iterations", C.c_int * 3), ("inner_iterations", C.c_int * 3),
                ("poisson_res_rel", C.c_double * 3), ("poisson_status", C.c_int * 3)]


_PP = C.POINTER(_dp)  # double**


def lib():
    """Load libimpact_b200.so (raises ImpactError when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImpactError(f"{LIB_PATH} is missing: build it with `python -m impact_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    i, d = C.c_int, C.c_double
    P = C.POINTER
    sigs = {
        "impact_b200_last_error": (C.c_char_p, []),
        "impact_b200_clear_error": (None, []),
        "impact_b200_version": (i, []),
        "impact_b200_set_stream": (None, [_vp]),
        "impact_b200_sync": (i, []),
        "impact_b200_axis_coords": (i, [i, d, i, _dp, _dp]),
        "impact_b200_axis_coeffs": (i, [i, _dp, _dp, P(AxisTables)]),
        "impact_b200_fd_exact": (i, [i, i, d, _dp]),
        "impact_b200_case_create": (i, [P(CaseDesc), P(Coeffs), P(_vp)]),
        "impact_b200_case_destroy": (i, [_vp]),
        "impact_b200_case_bytes": (C.c_longlong, [i, i, i, i]),
        "impact_b200_case_upload": (i, [_vp, i, _dp]),
        "impact_b200_case_download": (i, [_vp, i, _dp]),
        "impact_b200_case_upload_async": (i, [_vp, i, _dp, C.c_size_t, C.c_size_t, _vp]),
        "impact_b200_case_download_async": (i, [_vp, i, _dp, C.c_size_t, C.c_size_t, _vp]),
        "impact_b200_case_defer_pressure": (i, [_vp, _vp]),
        "impact_b200_case_set_inflow_waveform": (i, [_vp, i, _dp, _dp]),
        "impact_b200_case_snapshot": (i, [_vp, i, C.POINTER(i), C.POINTER(_dp), _vp]),
        "impact_b200_case_synchronize": (i, [_vp]),
        "impact_b200_case_set_labels": (i, [_vp, _u8p]),
        "impact_b200_case_set_markers": (i, [_vp, i, _dp, _u8p, C.c_double, i]),
        "impact_b200_case_ibm_interpolate": (i, [_vp, _dp]),
        "impact_b200_case_ibm_spread": (i, [_vp, _dp, _dp, i]),
        "impact_b200_case_field_ptr": (_vp, [_vp, i]),
        "impact_b200_case_stream": (_vp, [_vp]),
        "impact_b200_case_poisson": (i, [_vp, i, i, P(SolverParams), P(SolverResult)]),
        "impact_b200_case_step": (i, [_vp, P(StepParams), P(StepState), i]),
        "impact_b200_case_precond": (i, [_vp, i, i, P(SolverParams)]),
        "impact_b200_case_apply": (i, [_vp, i, i, i]),
        "impact_b200_batch_create": (i, [C.POINTER(_vp), i, C.POINTER(_vp)]),
        "impact_b200_batch_destroy": (i, [_vp]),
        "impact_b200_batch_step": (i, [_vp, C.POINTER(StepParams), C.POINTER(StepState), i]),
        "impact_b200_batch_size": (i, [_vp]),
        "impact_b200_batch_stream": (_vp, [_vp]),
        "impact_b200_case_mg_levels": (i, [_vp]),
        "impact_b200_jacobi_solve": (i, [i, i, i, i, i, i, d, _dp, _dp, _dp, _dp, _dp, i, d, i, _ip, _dp]),
        "impact_b200_jacobi_solve_bc": (i, [i, i, i, i, i, i, d, _dp, _dp, _dp, _dp, _dp, i, d, i, _ip, _dp,
                                            _u8p, i, i, i, i, d, d, d]),
        "impact_b200_product_scalar": (i, [i, i, i, _vp, _vp, _dp]),
        "impact_b200_product_scalar_noalloc": (i, [i, i, i, _vp, _vp, _dp]),
        "impact_b200_set_pressure_bc_plane": (i, [i]),
        "impact_b200_pressure_bc_plane": (i, []),
        "impact_b200_profile_enable": (None, [i]),
        "impact_b200_profile_reset": (None, []),
        "impact_b200_profile_read": (i, [i, P(C.c_longlong), _dp, _dp, P(C.c_char_p)]),
        "impact_b200_launch_count": (C.c_longlong, []),
        "impact_b200_case_kernel_bench": (i, [_vp, i, i, _dp]),
        "impact_b200_case_engine_bench": (i, [_vp, i, i, P(SolverParams), _dp, _dp]),
        # reference launcher FFI (every argument by reference)
        "gradient_launcher_": (None, [_ip] * 6 + [_PP] * 3),
        "divergence_launcher_": (None, [_ip] * 6 + [_PP] * 3),
        "divergence2_launcher_": (None, [_ip] * 6 + [_PP] * 5),
        "helmholtz_explicit_launcher_": (None, [_ip] * 7 + [_dp] + [_PP] * 5),
        "nonlinear_upwind_launcher_": (None, [_ip] * 6 + [_PP] * 5),
        "interpolate2_pre_vel_launcher_": (None, [_ip] * 6 + [_PP] * 3),
        "interpolate2_vel_pre_launcher_": (None, [_ip] * 6 + [_PP] * 3),
        "axpby_launcher_": (None, [_ip] * 3 + [_dp] * 2 + [_PP] * 3),
        "jor_launcher_": (None, [_ip] * 8 + [_dp] + [_PP] * 11),
        "get_ghost_launcher_": (None, [_ip] * 3 + [_PP] * 7),
        "pressure_bc_launcher_": (None, [_ip] * 7 + [_dp] * 3 + [_PP] * 2),
        "jacobi_launcher_": (None, [_ip] * 8 + [_dp] + [_PP] * 6),
        "product_dg_relax_launcher_": (None, [_ip] * 8 + [_PP] * 5),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return lib().impact_b200_last_error().decode()


def check(rc: int, what: str = ""):
    """Raise ImpactError with the library's message when rc != 0 (the message is then cleared,
    so that later calls do not report it again)."""
    if rc != 0:
        msg = last_error()
        lib().impact_b200_clear_error()
        raise ImpactError(f"{what}: {msg} (rc={rc})")


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "float64 C-contiguous array expected"
    return a.ctypes.data_as(_dp)


# Interior table widths (mod_dims.f90 ncb*(4)): 7 central, 6 gradient / divergence.
TABLE_WIDTH = {"cG": 6, "cD": 6, "cIpu": 6, "cIup": 6, "cNpU": 7, "cNpD": 7, "cNuU": 7, "cNuD": 7,
               "cp1": 7, "cpp": 7, "cuu": 7}


class Grid:
    """Coordinates and every coefficient table of a periodic grid with N = (N1, N2, N3) points.

    kinds[a] = 0 equidistant, 1 sinh-stretched.  Tables are numpy arrays in the reference layout.
    """

    def __init__(self, N, L=(1.0, 1.0, 1.0), kinds=(0, 0, 0)):
        self.N = tuple(int(n) for n in N)
        self.L = tuple(float(x) for x in L)
        self.kinds = tuple(int(k) for k in kinds)
        L_ = lib()
        self.xp, self.xu, self.tab = [], [], {n: [None] * 3 for n in list(TABLE_WIDTH) + ["cdg"]}
        self._axis = []
        for a in range(3):
            M = self.N[a]
            xp, xu = np.zeros(M + 7), np.zeros(M + 7)
            check(L_.impact_b200_axis_coords(M, self.L[a], self.kinds[a], _ptr(xp), _ptr(xu)), "axis_coords")
            t = AxisTables()
            for n, w in TABLE_WIDTH.items():
                arr = np.zeros(w * (M + 1))
                self.tab[n][a] = arr
                setattr(t, n, _ptr(arr))
            cdg = np.zeros(3 * M)
            self.tab["cdg"][a] = cdg
            t.cdg = _ptr(cdg)
            check(L_.impact_b200_axis_coeffs(M, _ptr(xp), _ptr(xu), C.byref(t)), "axis_coeffs")
            self.xp.append(xp)
            self.xu.append(xu)
            self._axis.append(t)
        self.coeffs = Coeffs()
        for a in range(3):
            self.coeffs.axis[a] = C.pointer(self._axis[a])
            self.coeffs.xp[a] = _ptr(self.xp[a])
            self.coeffs.xu[a] = _ptr(self.xu[a])
            self.coeffs.L[a] = self.L[a]

    @property
    def shape(self):
        N1, N2, N3 = self.N
        return (N3 + 7, N2 + 7, N1 + 7)

    @property
    def cells(self):
        return (self.N[0] - 1) * (self.N[1] - 1) * (self.N[2] - 1)

    def zeros(self, n=None):
        return np.zeros(self.shape if n is None else (n,) + self.shape)

    def interior(self, a):
        N1, N2, N3 = self.N
        return a[..., 4:N3 + 3, 4:N2 + 3, 4:N1 + 3]


def solver_params(tol_rel=1e-8, tol_abs_inf=0.0, max_it=2000, n_sweeps=4, omega=0.8, init_yes=0,
                  check_every=4, inner_tol_rel=1e-3, inner_max_it=0, precond=0, mg_down=4, mg_up=4,
                  mg_bottom=4, tile_kc=0, smooth_unfused=0, bottom_cheb=0) -> SolverParams:
    """precond 0: n_sweeps damped-Jacobi sweeps; 1: multigrid V-cycle (mg_down/up/bottom sweeps).
    tile_kc: z-planes per tile of the solver kernels (0: library default).  smooth_unfused: 1 runs
    every V-cycle sweep as its own launch instead of one fused kernel per smoothing phase.
    bottom_cheb: d > 0 replaces the coarsest level's Jacobi sweeps by d Chebyshev steps (fused
    schedule, coarsest level within the one-block tail)."""
    return SolverParams(tol_rel, tol_abs_inf, max_it, n_sweeps, omega, init_yes, check_every,
                        inner_tol_rel, inner_max_it, precond, mg_down, mg_up, mg_bottom, tile_kc, smooth_unfused,
                        bottom_cheb)


def step_params(Re=200.0, CFL=0.2, dtime_max=1e-2, dtime0=1e9, U0=1.0, T_pulse=1.0, level_pressure=1,
                explicit_fp32=0, **solver) -> StepParams:
    """explicit_fp32 (mixed-precision cases): rhs_vel as the FP32 pass instead of the FP64 one."""
    return StepParams(Re, CFL, dtime_max, dtime0, U0, T_pulse, level_pressure, solver_params(**solver),
                      int(explicit_fp32))


class Case:
    """One simulation case resident on one GPU (impact_b200_case_* of include/impact_b200.h)."""

    def __init__(self, grid: Grid, precision: int = 0, device: int = 0, stream=None):
        self.grid = grid
        self.precision = precision
        desc = CaseDesc(grid.N[0], grid.N[1], grid.N[2], precision, device, stream)
        h = _vp()
        check(lib().impact_b200_case_create(C.byref(desc), C.byref(grid.coeffs), C.byref(h)), "case_create")
        self._h = h
        self.state = StepState()

    def close(self):
        if self._h:
            lib().impact_b200_case_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def bytes_needed(N, precision=0) -> int:
        return int(lib().impact_b200_case_bytes(N[0], N[1], N[2], precision))

    def upload(self, field, host: np.ndarray):
        f = FIELDS[field] if isinstance(field, str) else field
        check(lib().impact_b200_case_upload(self._h, f, _ptr(np.ascontiguousarray(host))), "case_upload")

    def download(self, field, out: np.ndarray | None = None) -> np.ndarray:
        f = FIELDS[field] if isinstance(field, str) else field
        out = self.grid.zeros() if out is None else out
        check(lib().impact_b200_case_download(self._h, f, _ptr(out)), "case_download")
        return out

    def _range(self, what, a, first, count):
        if not (a.flags["C_CONTIGUOUS"] and a.dtype == np.float64 and a.shape == self.grid.shape):
            raise ValueError(what + ": host array must be C-contiguous float64 of the grid's shape")
        count = a.size - first if count is None else count
        if first < 0 or count < 0 or first + count > a.size:
            raise ValueError(what + ": element range outside the field")
        return first, count

    def upload_async(self, field, host: np.ndarray, stream: int = 0, first: int = 0, count: int | None = None):
        """Enqueue the copy of elements [first, first + count) (default: all) of `host` (C-contiguous
        float64 of the grid's shape, pinned for overlap) into the field on the CUDA stream handle
        `stream` (0: the case stream) and return at once; that range of `host` must stay alive and
        unchanged until the copy has completed."""
        f = FIELDS[field] if isinstance(field, str) else field
        first, count = self._range("upload_async", host, first, count)
        check(lib().impact_b200_case_upload_async(self._h, f, _ptr(host), first, count, C.c_void_p(stream or None)),
              "case_upload_async")

    def download_async(self, field, out: np.ndarray, stream: int = 0, first: int = 0, count: int | None = None):
        """Enqueue the copy of the field's elements [first, first + count) into `out` (as
        upload_async) and return at once."""
        f = FIELDS[field] if isinstance(field, str) else field
        first, count = self._range("download_async", out, first, count)
        check(lib().impact_b200_case_download_async(self._h, f, _ptr(out), first, count, C.c_void_p(stream or None)),
              "case_download_async")

    def defer_pressure(self, event: int):
        """The next step waits for the CUDA event handle `event` (e.g. torch.cuda.Event().cuda_event,
        recorded after an asynchronous pressure upload) only where it first reads the pressure; the
        event must stay alive until that step call has returned."""
        check(lib().impact_b200_case_defer_pressure(self._h, C.c_void_p(event)), "case_defer_pressure")

    def snapshot(self, fields, out, stream: int = 0):
        """Take device copies of `fields` now (in the case stream's order) and read them back into
        `out` (one C-contiguous float64 array of the grid's shape per field, pinned for overlap) on
        the CUDA stream handle `stream` (0: the case stream); returns at once.  `out` holds the
        snapshot once that stream has reached this point."""
        ids = [FIELDS[f] if isinstance(f, str) else int(f) for f in fields]
        if len(ids) != len(out):
            raise ValueError("snapshot: one output array per field")
        for a in out:
            if not (a.flags["C_CONTIGUOUS"] and a.dtype == np.float64 and a.shape == self.grid.shape):
                raise ValueError("snapshot: outputs must be C-contiguous float64 arrays of the grid's shape")
        fid = (C.c_int * len(ids))(*ids)
        ptrs = (_dp * len(out))(*[_ptr(a) for a in out])
        check(lib().impact_b200_case_snapshot(self._h, len(ids), fid, ptrs, C.c_void_p(stream or None)),
              "case_snapshot")

    def synchronize(self):
        """Wait until the case stream has finished its work."""
        check(lib().impact_b200_case_synchronize(self._h), "case_synchronize")

    def set_inflow_waveform(self, time=None, velocity=None):
        """Measured inflow of the label-5 voxels: nondimensional (time, velocity) pairs, times
        non-decreasing, the last one the pulse length (see impact_b200.ingest); None restores the
        default sinusoidal inflow."""
        if time is None:
            check(lib().impact_b200_case_set_inflow_waveform(self._h, 0, None, None), "case_set_inflow_waveform")
            return
        t = np.ascontiguousarray(time, dtype=np.float64)
        u = np.ascontiguousarray(velocity, dtype=np.float64)
        if t.ndim != 1 or t.shape != u.shape:
            raise ValueError("set_inflow_waveform: time and velocity must be 1-D arrays of one length")
        check(lib().impact_b200_case_set_inflow_waveform(self._h, t.size, _ptr(t), _ptr(u)), "case_set_inflow_waveform")

    def set_markers(self, yb, reach, delta_type=2, skip=None):
        """Immersed-boundary markers at positions yb (n, 3); skip: n flags of excluded markers;
        delta_type 1 cosine, 2 hat, 3 and 4 piecewise kernels of half-width reach / 2."""
        y = np.asarray(yb, dtype=np.float64)
        if y.ndim != 2 or y.shape[1] != 3:
            raise ValueError("set_markers: positions must be an (n, 3) array")
        flat = np.ascontiguousarray(y.T)
        sk = None
        if skip is not None:
            sk = np.ascontiguousarray(skip, dtype=np.uint8)
            if sk.shape != (y.shape[0],):
                raise ValueError("set_markers: one skip flag per marker")
            sk = sk.ctypes.data_as(_u8p)
        check(lib().impact_b200_case_set_markers(self._h, y.shape[0], _ptr(flat), sk, float(reach), int(delta_type)),
              "case_set_markers")
        self._markers = y.shape[0]  # only once the library holds this set

    def ibm_interpolate(self) -> np.ndarray:
        """Velocity of the resident fields at the markers, (n, 3)."""
        n = getattr(self, "_markers", 0)
        ub = np.zeros((3, n))
        check(lib().impact_b200_case_ibm_interpolate(self._h, _ptr(ub)), "case_ibm_interpolate")
        return ub.T.copy()

    def ibm_spread(self, fb, node_vol, into="rhs"):
        """Force density of the marker forces fb (n, 3) with node volumes node_vol (n,) into the
        fields rhs1..3 (into="rhs") or nl1..3 (into="nl"); returns the first field's name."""
        n = getattr(self, "_markers", 0)
        f = np.ascontiguousarray(np.asarray(fb, dtype=np.float64).reshape(n, 3).T)
        vol = np.ascontiguousarray(node_vol, dtype=np.float64).reshape(n)
        first = {"rhs": FIELDS["rhs1"], "nl": FIELDS["nl1"]}[into]
        check(lib().impact_b200_case_ibm_spread(self._h, _ptr(f), _ptr(vol), first), "case_ibm_spread")
        return into + "1"

    def set_labels(self, labels: np.ndarray):
        lb = np.ascontiguousarray(labels, dtype=np.uint8)
        check(lib().impact_b200_case_set_labels(self._h, lb.ctypes.data_as(_u8p)), "case_set_labels")

    def field_ptr(self, field) -> int:
        f = FIELDS[field] if isinstance(field, str) else field
        return lib().impact_b200_case_field_ptr(self._h, f)

    @property
    def stream(self):
        return lib().impact_b200_case_stream(self._h)

    def poisson(self, b="res", x="pre", params: SolverParams | None = None) -> SolverResult:
        params = solver_params() if params is None else params
        r = SolverResult()
        bi = FIELDS[b] if isinstance(b, str) else b
        xi = FIELDS[x] if isinstance(x, str) else x
        check(lib().impact_b200_case_poisson(self._h, bi, xi, C.byref(params), C.byref(r)), "case_poisson")
        return r

    @property
    def mg_levels(self) -> int:
        return lib().impact_b200_case_mg_levels(self._h)

    def precond(self, field_in="res", field_out="pre", params: SolverParams | None = None):
        """field_out = M field_in with the preconditioner of params (mixed-precision cases: the FP32
        preconditioner of the inner solve, on the input rounded to FP32)."""
        params = solver_params() if params is None else params
        fi = FIELDS[field_in] if isinstance(field_in, str) else field_in
        fo = FIELDS[field_out] if isinstance(field_out, str) else field_out
        check(lib().impact_b200_case_precond(self._h, fi, fo, C.byref(params)), "case_precond")

    def engine_bench(self, kind: int, iters: int = 10, params: SolverParams | None = None):
        """(ms per launch, algorithmic bytes per launch) of one Poisson-engine kernel kind"""
        params = solver_params(precond=1) if params is None else params
        ms, by = C.c_double(), C.c_double()
        check(lib().impact_b200_case_engine_bench(self._h, kind, iters, C.byref(params), C.byref(ms), C.byref(by)),
              "engine_bench")
        return ms.value, by.value

    def apply(self, field_in="pre", field_out="res", op: int = 0):
        """op 0: field_out = A field_in (product_div_grad); op 1: field_out = div(velocity);
        op 2: op 0 through the FP32 operator of the mixed solve"""
        fi = FIELDS[field_in] if isinstance(field_in, str) else field_in
        fo = FIELDS[field_out] if isinstance(field_out, str) else field_out
        check(lib().impact_b200_case_apply(self._h, op, fi, fo), "case_apply")

    def kernel_bench(self, kid: int, iters: int = 10) -> float:
        """average ms of one hot kernel launched iters times on the resident fields"""
        ms = C.c_double()
        check(lib().impact_b200_case_kernel_bench(self._h, kid, iters, C.byref(ms)), "kernel_bench")
        return ms.value

    def step(self, params: StepParams, nsteps: int = 1) -> StepState:
        check(lib().impact_b200_case_step(self._h, C.byref(params), C.byref(self.state), nsteps), "case_step")
        return self.state


class Batch:
    """Several cases of one device and precision advanced together (impact_b200_batch_*): one
    launch per operator of the pressure solve over all cases, graph-replayed iteration chunks.
    Each case keeps its own StepState (case.state), which the batch updates."""

    def __init__(self, cases):
        self.cases = list(cases)
        arr = (_vp * len(self.cases))(*[c._h for c in self.cases])
        h = _vp()
        check(lib().impact_b200_batch_create(arr, len(self.cases), C.byref(h)), "batch_create")
        self._h = h

    def close(self):
        if self._h:
            lib().impact_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, params, nsteps: int = 1):
        """params: one StepParams for all cases, or a list with one per case"""
        n = len(self.cases)
        plist = list(params) if isinstance(params, (list, tuple)) else [params] * n
        pa = (StepParams * n)(*plist)
        sa = (StepState * n)(*[c.state for c in self.cases])
        check(lib().impact_b200_batch_step(self._h, pa, sa, nsteps), "batch_step")
        for c, s in zip(self.cases, sa):
            C.memmove(C.byref(c.state), C.byref(s), C.sizeof(StepState))
        return [c.state for c in self.cases]

    @property
    def stream(self):
        return lib().impact_b200_batch_stream(self._h)


PROFILE_KERNELS = 19


def profile(enable: bool = True, reset: bool = True):
    """Turn the library's per-kernel CUDA-event timing on or off."""
    if reset:
        lib().impact_b200_profile_reset()
    lib().impact_b200_profile_enable(int(enable))


def profile_read():
    """{kernel name: (launches, total ms, algorithmic bytes)} of the profiled kernels."""
    out = {}
    for k in range(PROFILE_KERNELS):
        n, ms, by, nm = C.c_longlong(), C.c_double(), C.c_double(), C.c_char_p()
        check(lib().impact_b200_profile_read(k, C.byref(n), C.byref(ms), C.byref(by), C.byref(nm)), "profile_read")
        out[nm.value.decode()] = (n.value, ms.value, by.value)
    return out


def launch_count() -> int:
    return int(lib().impact_b200_launch_count())


def fd_exact(abl, n, deltaX0):
    cc = np.zeros(n)
    check(lib().impact_b200_fd_exact(abl, n, float(deltaX0), _ptr(cc)), "fd_exact")
    return cc


def product_scalar(N, a_dev: int, b_dev: int) -> float:
    out = C.c_double()
    check(lib().impact_b200_product_scalar(N[0], N[1], N[2], a_dev, b_dev, C.byref(out)), "product_scalar")
    return out.value


def product_scalar_noalloc(N, a_dev: int, b_dev: int) -> float:
    """product_scalar without any device allocation (fixed library scratch; see the C header)."""
    out = C.c_double()
    check(lib().impact_b200_product_scalar_noalloc(N[0], N[1], N[2], a_dev, b_dev, C.byref(out)),
          "product_scalar_noalloc")
    return out.value


def set_pressure_bc_plane(mode: int):
    """Plane of the inlet / first-outlet pressure condition (pressure_bc_launcher_ and the JOR solve
    with the CT condition): 0 (default) the Fortran test k == k_start_index - 1 of
    apply_pressure_BC_CT (usr_func.f90:857-897); 1 the plane the reference GPU kernel sets,
    k_start_index - 4 (set_pressure_BC_kernel.cu:26)."""
    check(lib().impact_b200_set_pressure_bc_plane(int(mode)), "set_pressure_bc_plane")


def pressure_bc_plane() -> int:
    return int(lib().impact_b200_pressure_bc_plane())


def jacobi_solve(grid: Grid, rel: np.ndarray, bb: np.ndarray, omega=0.8, mode_j=20, tol_abs_inf=0.0,
                 max_sweeps=100000, M=None, labels=None, k_start_index=0, type_ids=(1, 1, 0),
                 pressures=(0.0, 0.0, 0.0)):
    """device_jacobi_solver replacement on host arrays; returns (sweeps, res_inf).  With labels,
    the CT pressure condition of the third substep is applied at the start of every iteration
    (pressures: inlet, outlet, second outlet, already multiplied by (aRK + bRK) dt)."""
    N1, N2, N3 = grid.N
    M1, M2, M3 = M if M is not None else grid.N
    sw, ri = C.c_int(), C.c_double()
    c = grid.tab["cdg"]
    args = (N1, N2, N3, M1, M2, M3, omega, _ptr(c[0]), _ptr(c[1]), _ptr(c[2]), _ptr(rel), _ptr(bb), mode_j,
            tol_abs_inf, max_sweeps, C.byref(sw), C.byref(ri))
    if labels is None:
        check(lib().impact_b200_jacobi_solve(*args), "jacobi_solve")
    else:
        lb = np.ascontiguousarray(labels, dtype=np.uint8)
        if lb.shape != grid.shape:
            raise ValueError("jacobi_solve: labels must have the padded field shape")
        check(lib().impact_b200_jacobi_solve_bc(*args, lb.ctypes.data_as(_u8p), k_start_index, *type_ids,
                                                *pressures), "jacobi_solve_bc")
    return sw.value, ri.value


class launchers:
    """The reference's launcher FFI on device pointers (ints), every argument passed by reference."""

    @staticmethod
    def call(name, *args):
        """args: ('i', int) | ('d', float as FP64) | ('f', float as FP32) | ('p', device pointer);
        the _sp_ launchers take their scalars as 'f'."""
        conv = []
        keep = []
        for kind, v in args:
            if kind == "i":
                o = C.c_int(int(v))
            elif kind == "d":
                o = C.c_double(float(v))
            elif kind == "f":
                o = C.c_float(float(v))
            else:
                o = C.cast(C.c_void_p(int(v)), _dp)
            keep.append(o)
            conv.append(C.byref(o))
        getattr(lib(), name)(*conv)
        err = last_error()
        if err:
            lib().impact_b200_clear_error()
            raise ImpactError(f"{name}: {err}")

    @staticmethod
    def sync():
        check(lib().impact_b200_sync(), "sync")
