"""ctypes front end of the CPU FP64 oracle (liboracle.so built from impact_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py``.  The CUDA product never imports it.

Fields are numpy float64 arrays of shape (N3+7, N2+7, N1+7) -- C order, i.e. the same
memory as IMPACT's column-major ``phi(-3:N1+3, -3:N2+3, -3:N3+3)`` (mod_vars.f90:476-518).
``interior(a)`` is the view of the unique periodic points 1..N-1 per axis.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


class OrcCoeffs(C.Structure):
    _fields_ = [(name, _dp * 3) for name in (
        "cG", "cD", "cIpu", "cIup", "cNpU", "cNpD", "cNuU", "cNuD", "cp1", "cpp", "cuu", "cdg")]


class OrcSolverOpts(C.Structure):
    _fields_ = [("tol_rel", C.c_double), ("tol_abs_inf", C.c_double), ("max_it", C.c_int),
                ("n_sweeps", C.c_int), ("omega", C.c_double), ("init_yes", C.c_int), ("precond", C.c_int),
                ("mg", C.c_void_p), ("mg_down", C.c_int), ("mg_up", C.c_int), ("mg_bottom", C.c_int)]


class OrcSolverResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("res_inf", C.c_double),
                ("res_two", C.c_double), ("b_two", C.c_double)]


MG_MAX = 15


class OrcMG(C.Structure):
    _fields_ = [("n_grids", C.c_int), ("M", (C.c_int * 3) * MG_MAX), ("ratio", (C.c_int * 3) * MG_MAX),
                ("xp", (_dp * 3) * MG_MAX), ("xu", (_dp * 3) * MG_MAX), ("cdg", (_dp * 3) * MG_MAX),
                ("cI", (_dp * 3) * MG_MAX), ("f", (_dp * 3) * MG_MAX)]


class OrcStepParams(C.Structure):
    _fields_ = [("Re", C.c_double), ("CFL", C.c_double), ("dtime_max", C.c_double),
                ("dtime0", C.c_double), ("U0", C.c_double), ("T_pulse", C.c_double),
                ("level_pressure", C.c_int), ("poisson", OrcSolverOpts)]


class OrcStepState(C.Structure):
    _fields_ = [("time", C.c_double), ("dtime", C.c_double), ("timestep", C.c_int),
                ("poisson_iterations", C.c_int * 3), ("poisson_res_rel", C.c_double * 3),
                ("poisson_status", C.c_int * 3)]


def build():
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        i, d = C.c_int, C.c_double
        P = C.POINTER
        sig = {
            "orc_coords": (None, [i, d, i, _dp, _dp]),
            "orc_fd_exact": (i, [i, i, d, _dp]),
            "orc_diff_coeffs": (i, [i, i, i, i, i, i, i, _dp, _dp, _dp]),
            "orc_get_stencil": (None, [i, _dp, _dp, _dp]),
            "orc_stability_limits": (None, [_dp]),
            "orc_set_threads": (i, [i]),
            "orc_exchange": (None, [i, i, i, i, _dp]),
            "orc_gradient": (None, [i, i, i, i, P(OrcCoeffs), _dp, _dp]),
            "orc_divergence": (None, [i, i, i, i, P(OrcCoeffs), _dp, _dp]),
            "orc_divergence2": (None, [i, i, i, P(OrcCoeffs), _dp, _dp, _dp, _dp]),
            "orc_helmholtz": (None, [i, i, i, i, P(OrcCoeffs), d, _dp, _dp]),
            "orc_interpolate_pre_vel": (None, [i, i, i, i, P(OrcCoeffs), _dp, _dp]),
            "orc_interpolate_vel_pre": (None, [i, i, i, i, P(OrcCoeffs), _dp, _dp]),
            "orc_nonlinear_upwind": (None, [i, i, i, i, P(OrcCoeffs), _dp, _dp, _dp]),
            "orc_nonlinear": (None, [i, i, i, i, P(OrcCoeffs), _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_axpby": (None, [i, i, i, d, d, _dp, _dp, _dp]),
            "orc_product_div_grad": (None, [i, i, i, P(OrcCoeffs), _dp, _dp, _dp]),
            "orc_product_dg_relax": (None, [i, i, i, P(OrcCoeffs), _dp, _dp]),
            "orc_jacobi": (None, [i, i, i, P(OrcCoeffs), i, i, d, _dp, _dp, _dp]),
            "orc_pressure_bc": (None, [i, i, i, _u8p, i, d, d, d, _dp]),
            "orc_product_scalar": (d, [i, i, i, _dp, _dp]),
            "orc_norms": (None, [i, i, i, _dp, _dp, _dp]),
            "orc_bicgstab": (None, [i, i, i, P(OrcCoeffs), P(OrcSolverOpts), _dp, _dp, _dp,
                                    P(OrcSolverResult)]),
            "orc_get_dtime": (d, [i, i, i, P(OrcCoeffs), _dp, d, d, d, _dp, _dp]),
            "orc_mg_build": (i, [i, i, i, P(_dp), P(_dp), _dp, i, P(OrcMG)]),
            "orc_mg_free": (None, [P(OrcMG)]),
            "orc_mg_vcycle": (None, [P(OrcMG), i, i, i, d, _dp, _dp, _dp]),
            "orc_bicgstab_mg": (None, [i, i, i, P(OrcCoeffs), P(OrcMG), P(OrcSolverOpts), i, i, i, _dp, _dp, _dp,
                                       P(OrcSolverResult)]),
            "orc_mask_forcing": (None, [i, i, i, _u8p, d, _dp]),
            "orc_level_pressure": (None, [i, i, i, _dp]),
            "orc_ibm_delta": (d, [i, d, d]),
            "orc_ibm_interpolate": (None, [i, i, i, P(_dp), P(_dp), _dp, i, d, i, _dp, _u8p, _dp, _dp]),
            "orc_ibm_spread": (None, [i, i, i, P(_dp), P(_dp), _dp, i, d, i, _dp, _u8p, _dp, _dp, _dp]),
            "orc_time_step": (None, [i, i, i, P(OrcCoeffs), P(OrcStepParams), _dp, _u8p, _dp,
                                     _dp, _dp, _dp, P(OrcStepState)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def u8ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u8p)


# Interior stencil widths of IMPACT (mod_dims.f90 ncb*c/g/d last entries; mod_vars.f90:157-214).
N_CENTRAL, N_GRAD, N_DIV = 7, 6, 6
B_LO, B_HI, D_LO, D_HI, G_LO, G_HI = -3, 3, -3, 2, -2, 3


class Grid:
    """Coordinates and every coefficient table of one periodic IMPACT grid (oracle side).

    N = (N1, N2, N3) are IMPACT's point counts (cells = N - 1 per periodic axis);
    kinds[a] = 0 equidistant, 1 sinh-stretched (x(s) = L/2 (1 + sinh(2(s/(N-1) - 1/2))/sinh 1)).
    Follows FD_coeffs (mod_coeffs.f90:37-112) and get_stencil (mod_coeffs.f90:1048).
    """

    def __init__(self, N, L=(1.0, 1.0, 1.0), kinds=(0, 0, 0)):
        self.N = tuple(int(n) for n in N)
        self.L = tuple(float(x) for x in L)
        self.kinds = tuple(int(k) for k in kinds)
        lb = lib()
        self.xp, self.xu, self.tab = [], [], {}
        names = ("cG", "cD", "cIpu", "cIup", "cNpU", "cNpD", "cNuU", "cNuD", "cp1", "cpp", "cuu", "cdg")
        for n in names:
            self.tab[n] = [None, None, None]
        for a in range(3):
            M = self.N[a]
            xp = np.zeros(M + 7)
            xu = np.zeros(M + 7)
            lb.orc_coords(M, self.L[a], self.kinds[a], ptr(xp), ptr(xu))
            self.xp.append(xp)
            self.xu.append(xu)

            def dc(abl, upw, gt, lo, hi, n, xC, xE):
                cc = np.zeros((M + 1) * (hi - lo + 1))
                rc = lb.orc_diff_coeffs(abl, upw, gt, M, lo, hi, n, ptr(xC), ptr(xE), ptr(cc))
                if rc != 0:
                    raise RuntimeError(f"orc_diff_coeffs failed ({rc})")
                return cc

            self.tab["cNpD"][a] = dc(1, -1, 0, B_LO, B_HI, N_CENTRAL, xp, xp)
            self.tab["cNpU"][a] = dc(1, 1, 0, B_LO, B_HI, N_CENTRAL, xp, xp)
            self.tab["cNuD"][a] = dc(1, -1, 1, B_LO, B_HI, N_CENTRAL, xu, xu)
            self.tab["cNuU"][a] = dc(1, 1, 1, B_LO, B_HI, N_CENTRAL, xu, xu)
            self.tab["cp1"][a] = dc(1, 0, 0, B_LO, B_HI, N_CENTRAL, xp, xp)
            self.tab["cpp"][a] = dc(2, 0, 0, B_LO, B_HI, N_CENTRAL, xp, xp)
            self.tab["cuu"][a] = dc(2, 0, 1, B_LO, B_HI, N_CENTRAL, xu, xu)
            self.tab["cG"][a] = dc(1, 0, 2, G_LO, G_HI, N_GRAD, xp, xu)
            self.tab["cD"][a] = dc(1, 0, 3, D_LO, D_HI, N_DIV, xu, xp)
            self.tab["cIpu"][a] = dc(0, 0, 2, G_LO, G_HI, N_GRAD, xp, xu)
            self.tab["cIup"][a] = dc(0, 0, 3, D_LO, D_HI, N_DIV, xu, xp)
            cdg = np.zeros(3 * M)
            lb.orc_get_stencil(M, ptr(xp), ptr(xu), ptr(cdg))
            self.tab["cdg"][a] = cdg
        self.c = OrcCoeffs()
        for n in names:
            setattr(self.c, n, (_dp * 3)(*[ptr(t) for t in self.tab[n]]))
        self.stab = np.zeros(41)
        lb.orc_stability_limits(ptr(self.stab))

    # ---- fields ----
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

    def random(self, seed, n=None, lo=-1.0, hi=1.0):
        rng = np.random.default_rng(seed)
        f = self.zeros(n)
        self.interior(f)[...] = rng.uniform(lo, hi, size=self.interior(f).shape)
        return f

    def fill_ghosts(self, a):
        """Periodic ghost fill of a field (all three directions)."""
        lb = lib()
        for d in (1, 2, 3):
            lb.orc_exchange(d, *self.N, ptr(a))
        return a

    # ---- divergence metric of the reference's in-code check ----
    def divergence_weight(self):
        """weight(i,j,k) = 1 / (sum_l |cDu1(l,i)| + sum_l |cDv2(l,j)| + sum_l |cDw3(l,k)|) at the
        unique pressure points, shape (N3-1, N2-1, N1-1) (mod_coeffs.f90:2242-2262; the corner
        zeroing of :2363 applies to walls only, never to a periodic box)."""
        s = []
        for a in range(3):
            c = self.tab["cD"][a].reshape(self.N[a] + 1, N_DIV)
            s.append(np.abs(c[1:self.N[a]]).sum(axis=1))
        return 1.0 / (s[2][:, None, None] + s[1][None, :, None] + s[0][None, None, :])

    def test_divergence(self, vel, where=None):
        """(max |div2(vel)|, max |div2(vel) * weight|) over the unique pressure points, as the
        reference's test_divergence prints them (mod_test.f90:300-345); `where` (bool, interior
        shape) restricts both maxima to a subset of the points."""
        d = self.interior(self.divergence2(vel[0], vel[1], vel[2]))
        w = self.divergence_weight()
        a, b = np.abs(d), np.abs(d * w)
        if where is not None:
            a, b = a[where], b[where]
        return float(a.max()), float(b.max())

    # ---- operators ----
    def gradient(self, m, phi, out=None):
        out = self.zeros() if out is None else out
        lib().orc_gradient(m, *self.N, C.byref(self.c), ptr(phi), ptr(out))
        return out

    def divergence(self, m, phi, div):
        lib().orc_divergence(m, *self.N, C.byref(self.c), ptr(phi), ptr(div))
        return div

    def divergence2(self, u, v, w, out=None):
        out = self.zeros() if out is None else out
        lib().orc_divergence2(*self.N, C.byref(self.c), ptr(u), ptr(v), ptr(w), ptr(out))
        return out

    def helmholtz(self, m, multL, vel, nl):
        lib().orc_helmholtz(m, *self.N, C.byref(self.c), multL, ptr(vel), ptr(nl))
        return nl

    def interpolate_pre_vel(self, m, phi, out=None):
        out = self.zeros() if out is None else out
        lib().orc_interpolate_pre_vel(m, *self.N, C.byref(self.c), ptr(phi), ptr(out))
        return out

    def interpolate_vel_pre(self, m, phi, out=None):
        out = self.zeros() if out is None else out
        lib().orc_interpolate_vel_pre(m, *self.N, C.byref(self.c), ptr(phi), ptr(out))
        return out

    # ---- immersed boundary transfers (mod_ibm.f90) ----
    def _ibm_args(self, yb, skip):
        yb = np.asfortranarray(yb, dtype=np.float64)
        n = yb.shape[0]
        flat = np.ascontiguousarray(yb.T)  # (3, n): all x, then all y, then all z
        sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.uint8)
        xp = (_dp * 3)(*[ptr(a) for a in self.xp])
        xu = (_dp * 3)(*[ptr(a) for a in self.xu])
        L = np.array(self.L)
        return n, flat, sk, xp, xu, L

    def ibm_interpolate(self, yb, vel, delta_type, reach, skip=None):
        """interpolate_vel_to_ib: marker velocities (n, 3) from the velocity fields vel (3, shape)."""
        n, flat, sk, xp, xu, L = self._ibm_args(yb, skip)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        ub = np.zeros((3, n))
        lib().orc_ibm_interpolate(*self.N, xp, xu, ptr(L), delta_type, reach, n, ptr(flat),
                                  None if sk is None else u8ptr(sk), ptr(vel), ptr(ub))
        return ub.T.copy()

    def ibm_spread(self, yb, fb, node_vol, delta_type, reach, skip=None):
        """spread_force_dens_to_vel_grid: force density fields (3, shape) from marker forces (n, 3)."""
        n, flat, sk, xp, xu, L = self._ibm_args(yb, skip)
        f = np.ascontiguousarray(np.asarray(fb, dtype=np.float64).T)
        vol = np.ascontiguousarray(node_vol, dtype=np.float64)
        fd = self.zeros(3)
        lib().orc_ibm_spread(*self.N, xp, xu, ptr(L), delta_type, reach, n, ptr(flat),
                             None if sk is None else u8ptr(sk), ptr(f), ptr(vol), ptr(fd))
        return fd

    def nonlinear_upwind(self, cid, pp, vel, nl):
        lib().orc_nonlinear_upwind(cid, *self.N, C.byref(self.c), ptr(pp), ptr(vel), ptr(nl))
        return nl

    def nonlinear(self, m, vel_m, w1, w2, w3, out=None):
        out = self.zeros() if out is None else out
        pp = self.zeros()
        lib().orc_nonlinear(m, *self.N, C.byref(self.c), ptr(vel_m), ptr(w1), ptr(w2), ptr(w3),
                            ptr(pp), ptr(out))
        return out

    def axpby(self, a, b, x, y, z):
        lib().orc_axpby(*self.N, a, b, ptr(x), ptr(y), ptr(z))
        return z

    def product_div_grad(self, phi, out=None):
        out = self.zeros() if out is None else out
        dig = self.zeros()
        lib().orc_product_div_grad(*self.N, C.byref(self.c), ptr(phi), ptr(dig), ptr(out))
        return out

    def product_dg_relax(self, phi, out=None):
        out = self.zeros() if out is None else out
        lib().orc_product_dg_relax(*self.N, C.byref(self.c), ptr(phi), ptr(out))
        return out

    def jacobi(self, bb, rel, n_relax, omega, init_yes=False):
        comp = self.zeros()
        lib().orc_jacobi(*self.N, C.byref(self.c), int(init_yes), n_relax, omega, ptr(bb), ptr(rel),
                         ptr(comp))
        return rel

    def pressure_bc(self, label, k_start_index, p_in, p_out, p_out2, rel):
        lib().orc_pressure_bc(*self.N, u8ptr(label), k_start_index, p_in, p_out, p_out2, ptr(rel))
        return rel

    def dot(self, a, b):
        return lib().orc_product_scalar(*self.N, ptr(a), ptr(b))

    def norms(self, a):
        ni, n2 = C.c_double(), C.c_double()
        lib().orc_norms(*self.N, ptr(a), C.byref(ni), C.byref(n2))
        return ni.value, n2.value

    def bicgstab(self, bb, phi, tol_rel=1e-8, tol_abs_inf=0.0, max_it=1000, n_sweeps=4, omega=0.8,
                 init_yes=False):
        o = OrcSolverOpts(tol_rel, tol_abs_inf, max_it, n_sweeps, omega, int(init_yes), 0, None, 4, 4, 4)
        work = self.zeros(9)
        r = OrcSolverResult()
        lib().orc_bicgstab(*self.N, C.byref(self.c), C.byref(o), ptr(bb), ptr(phi), ptr(work),
                           C.byref(r))
        return r

    def multigrid(self, n_grids_limit=15):
        """Build the multigrid hierarchy of this grid (mod_setup.f90:95-143)."""
        return MG(self, n_grids_limit)

    def get_dtime(self, vel, Re, CFL, dtime_max):
        work = self.zeros(3)
        return lib().orc_get_dtime(*self.N, C.byref(self.c), ptr(self.stab), Re, CFL, dtime_max,
                                   ptr(vel), ptr(work))

    def mask_forcing(self, label, u_in, vel):
        lib().orc_mask_forcing(*self.N, u8ptr(label), u_in, ptr(vel))
        return vel

    def level_pressure(self, pre):
        lib().orc_level_pressure(*self.N, ptr(pre))
        return pre

    def time_step(self, params: OrcStepParams, label, vel, nl, pre, state: OrcStepState, scratch=None):
        scratch = self.zeros(17) if scratch is None else scratch
        lib().orc_time_step(*self.N, C.byref(self.c), C.byref(params), ptr(self.stab), u8ptr(label),
                            ptr(vel), ptr(nl), ptr(pre), ptr(scratch), C.byref(state))
        return state


class MG:
    """Multigrid hierarchy of a periodic oracle grid (levels, coordinates, cdg, cI, level fields)."""

    def __init__(self, grid: "Grid", n_grids_limit=15):
        self.grid = grid
        self.s = OrcMG()
        xp = (_dp * 3)(*[ptr(a) for a in grid.xp])
        xu = (_dp * 3)(*[ptr(a) for a in grid.xu])
        L = np.array(grid.L, dtype=np.float64)
        rc = lib().orc_mg_build(*grid.N, xp, xu, ptr(L), n_grids_limit, C.byref(self.s))
        if rc != 0:
            raise RuntimeError("orc_mg_build failed")

    @property
    def n_grids(self):
        return self.s.n_grids

    def level_sizes(self):
        return [tuple(self.s.M[g][m] for m in range(3)) for g in range(self.n_grids)]

    def level_table(self, name, g, m):
        M = self.s.M[g][m]
        n = {"xp": M + 7, "xu": M + 7, "cdg": 3 * M, "cI": 2 * (M + 1)}[name]
        return np.ctypeslib.as_array(getattr(self.s, name)[g][m], shape=(n,)).copy()

    def vcycle(self, bb, phi, n_down=4, n_up=4, n_bottom=4, omega=0.98):
        work = self.grid.zeros()
        lib().orc_mg_vcycle(C.byref(self.s), n_down, n_up, n_bottom, omega, ptr(bb), ptr(phi), ptr(work))
        return phi

    def bicgstab(self, bb, phi, tol_rel=1e-8, max_it=200, omega=0.98, n_down=4, n_up=4, n_bottom=4,
                 init_yes=False):
        g = self.grid
        o = OrcSolverOpts(tol_rel, 0.0, max_it, 1, omega, int(init_yes), 0, None, n_down, n_up, n_bottom)
        work = g.zeros(9)
        r = OrcSolverResult()
        lib().orc_bicgstab_mg(*g.N, C.byref(g.c), C.byref(self.s), C.byref(o), n_down, n_up, n_bottom, ptr(bb),
                              ptr(phi), ptr(work), C.byref(r))
        return r

    def __del__(self):
        try:
            lib().orc_mg_free(C.byref(self.s))
        except Exception:
            pass


def step_params(Re=200.0, CFL=0.2, dtime_max=1e-2, dtime0=1e9, U0=1.0, T_pulse=1.0, level_pressure=1,
                tol_rel=1e-8, max_it=2000, n_sweeps=4, omega=0.8, mg=None, mg_down=4, mg_up=4, mg_bottom=4):
    """mg: an MG hierarchy (Grid.multigrid()) selects the V-cycle preconditioner."""
    o = OrcSolverOpts(tol_rel, 0.0, max_it, n_sweeps, omega, 0, 1 if mg is not None else 0,
                      C.cast(C.pointer(mg.s), C.c_void_p) if mg is not None else None, mg_down, mg_up, mg_bottom)
    p = OrcStepParams(Re, CFL, dtime_max, dtime0, U0, T_pulse, level_pressure, o)
    p._keep = mg
    return p


def set_threads(n: int) -> int:
    """OpenMP threads of the oracle's loops (n <= 0: query); returns the threads in use."""
    return int(lib().orc_set_threads(int(n)))


def fd_exact(abl, n, deltaX0):
    cc = np.zeros(n)
    rc = lib().orc_fd_exact(abl, n, float(deltaX0), ptr(cc))
    if rc != 0:
        raise ValueError("bad stencil")
    return cc
