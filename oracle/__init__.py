"""ctypes wrapper of the CPU FP64 oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker or the timed CPU baseline.  The
product (cup3d_b200) never imports it.  See oracle.h for what it restates and
how it is pinned.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)
_L = C.POINTER(C.c_int64)
_F = C.POINTER(C.c_float)
_lib = None

SIG = {
    "orc_mesh_create": (C.c_void_p, [C.c_int, _I, _I, _I, C.c_int, _I, C.c_double]),
    "orc_mesh_destroy": (None, [C.c_void_p]),
    "orc_mesh_nb": (C.c_int, [C.c_void_p]),
    "orc_mesh_h": (C.c_double, [C.c_void_p, C.c_int]),
    "orc_mesh_hmin": (C.c_double, [C.c_void_p]),
    "orc_mesh_faces": (None, [C.c_void_p, _I, _I]),
    "orc_poisson_nnz": (C.c_int64, [C.c_void_p, C.c_int]),
    "orc_poisson_csr": (None, [C.c_void_p, C.c_int, _L, _L, _D]),
    "orc_poisson_apply": (None, [C.c_void_p, C.c_int, _D, _D]),
    "orc_pinv": (None, [_D]),
    "orc_precond_pinv": (None, [C.c_void_p, _D, _D, _D]),
    "orc_precond_cg": (None, [C.c_void_p, _D, _D]),
    "orc_bicgstab_gpu": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _D, C.c_double, C.c_double, C.c_int,
                                   C.c_int, _D]),
    "orc_bicgstab_pipelined": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _D, C.c_double, C.c_double,
                                         C.c_int, _D]),
    "orc_fill_lab": (None, [C.c_void_p, _D, C.c_int, C.c_int, C.c_int, C.c_int, _D]),
    "orc_max_u": (C.c_double, [C.c_void_p, _D, _D]),
    "orc_dt": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]),
    "orc_advect_diffuse": (None, [C.c_void_p, _D, _D, C.c_double, C.c_double, _D, C.c_int]),
    "orc_advect_rhs": (None, [C.c_void_p, _D, _D, C.c_double, C.c_double, _D, C.c_int, C.c_double]),
    "orc_penalize": (None, [C.c_void_p, _D, _D, _I, C.c_int, _D, _D, _D, C.c_double, C.c_double, C.c_int,
                            _D]),
    "orc_pressure_project": (None, [C.c_void_p, _D, _D, _D, _I, C.c_int, _D, _D, C.c_double, C.c_int, C.c_int,
                                    C.c_int, C.c_double, C.c_double, _D, _D]),
    "orc_pressure_rhs": (None, [C.c_void_p, _D, _D, _D, _I, C.c_int, _D, _D, C.c_double, C.c_int, _D]),
    "orc_grad_update": (None, [C.c_void_p, _D, _D, C.c_double]),
    "orc_dissipation": (None, [C.c_void_p, _D, _D, _D, C.c_double, _D]),
    "orc_create_obstacle": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D, _I, _I, _D, _D, _D]),
    "orc_obstacle_surface": (None, [C.c_void_p, C.c_int, _D, _D, _D, C.c_int, _I, _D, _D]),
    "orc_compute_forces": (C.c_int, [C.c_void_p, _D, _D, _D, C.c_int, _I, _D, _D, C.c_double, _D, _D]),
    "orc_adapt_indicator": (None, [C.c_void_p, _D, _D, C.c_int, C.c_int, C.c_double, C.c_double, _D]),
    "orc_adapt_leaves": (C.c_int, [C.c_void_p, _D, C.c_double, C.c_double, _I, C.c_int]),
    "orc_adapt_transfer": (None, [C.c_void_p, C.c_void_p, _D, C.c_int, C.c_int, _D]),
    "orc_cnn_nparam": (C.c_int, [C.c_int]),
    "orc_cnn_fwd_grad": (None, [C.c_int, C.c_int, _D, _F, _F, _F, _D, _D]),
}


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
        L = C.CDLL(str(LIB_PATH))
        for k, (r, a) in SIG.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _i(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


def _f(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


class Mesh:
    """Oracle mesh over a leaf list given in the caller's block order."""

    def __init__(self, level, index, bpd, level_max, bc, extent):
        self.level = np.ascontiguousarray(level, np.int32)
        self.index = np.ascontiguousarray(np.asarray(index).reshape(-1), np.int32)
        bpd = np.ascontiguousarray(bpd, np.int32)
        bc = np.ascontiguousarray(bc, np.int32)
        p = lib().orc_mesh_create(len(self.level), _i(self.level), _i(self.index), _i(bpd), level_max, _i(bc),
                                  float(extent))
        if not p:
            raise ValueError("oracle rejected the mesh")
        self._p = C.c_void_p(p)
        self.nb = len(self.level)
        self.h = np.array([lib().orc_mesh_h(self._p, b) for b in range(self.nb)])
        self.hmin = lib().orc_mesh_hmin(self._p)

    def __del__(self):
        if getattr(self, "_p", None):
            lib().orc_mesh_destroy(self._p)
            self._p = None

    @property
    def n(self):
        return self.nb * 512

    def faces(self):
        k = np.zeros(6 * self.nb, np.int32)
        n = np.zeros(24 * self.nb, np.int32)
        lib().orc_mesh_faces(self._p, _i(k), _i(n))
        return k.reshape(self.nb, 6), n.reshape(self.nb, 6, 4)

    # Poisson
    def csr(self, mean_constraint=1):
        nnz = lib().orc_poisson_nnz(self._p, mean_constraint)
        rp = np.zeros(self.n + 1, np.int64)
        col = np.zeros(nnz, np.int64)
        val = np.zeros(nnz, np.float64)
        lib().orc_poisson_csr(self._p, mean_constraint, rp.ctypes.data_as(_L), col.ctypes.data_as(_L), _d(val))
        return rp, col, val

    def apply(self, x, mean_constraint=1):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        lib().orc_poisson_apply(self._p, mean_constraint, _d(x), _d(y))
        return y

    def precond_pinv(self, x, P=None):
        if P is None:
            P = pinv()
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        lib().orc_precond_pinv(self._p, _d(P), _d(x), _d(y))
        return y

    def precond_cg(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        lib().orc_precond_cg(self._p, _d(x), _d(y))
        return y

    def bicgstab_gpu(self, b, x0=None, tol=1e-6, tol_rel=1e-4, mean_constraint=1, precond=0, max_restarts=100,
                     max_iter=1000):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
        st = np.zeros(5)
        lib().orc_bicgstab_gpu(self._p, mean_constraint, precond, _d(b), _d(x), tol, tol_rel, max_restarts,
                               max_iter, _d(st))
        return x, dict(iterations=int(st[0]), restarts=int(st[1]), err_init=st[2], err_final=st[3],
                       converged=bool(st[4]))

    def bicgstab_pipelined(self, b, x0=None, tol=1e-6, tol_rel=1e-4, mean_constraint=1, precond=1,
                           max_iter=1000):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
        st = np.zeros(5)
        lib().orc_bicgstab_pipelined(self._p, mean_constraint, precond, _d(b), _d(x), tol, tol_rel, max_iter,
                                     _d(st))
        return x, dict(iterations=int(st[0]), restarts=int(st[1]), err_init=st[2], err_final=st[3],
                       converged=bool(st[4]))

    def lab(self, field, ncomp, G, block, vector_bc):
        f = np.ascontiguousarray(field, np.float64)
        W = 8 + 2 * G
        out = np.zeros(ncomp * W ** 3)
        lib().orc_fill_lab(self._p, _d(f), ncomp, G, block, int(vector_bc), _d(out))
        return out.reshape(ncomp, W, W, W)

    # operators
    def max_u(self, vel, uinf=(0, 0, 0)):
        u = np.ascontiguousarray(uinf, np.float64)
        return lib().orc_max_u(self._p, _d(np.ascontiguousarray(vel, np.float64)), _d(u))

    def advect_diffuse(self, vel, dt, nu, uinf=(0, 0, 0), scheme=0):
        vel = np.array(vel, np.float64)
        tmp = np.zeros_like(vel)
        u = np.ascontiguousarray(uinf, np.float64)
        lib().orc_advect_diffuse(self._p, _d(vel), _d(tmp), dt, nu, _d(u), scheme)
        return vel

    def advect_rhs(self, vel, dt, nu, uinf=(0, 0, 0), scheme=0, coef=1.0):
        vel = np.ascontiguousarray(vel, np.float64)
        tmp = np.zeros_like(vel)
        u = np.ascontiguousarray(uinf, np.float64)
        lib().orc_advect_rhs(self._p, _d(vel), _d(tmp), dt, nu, _d(u), scheme, coef)
        return tmp

    def penalize(self, vel, chi, slot, chi_o, udef_o, kin, dt, lam=1e6, implicit=1):
        vel = np.array(vel, np.float64)
        F = np.zeros(6)
        lib().orc_penalize(self._p, _d(vel), _d(np.ascontiguousarray(chi, np.float64)),
                           _i(np.ascontiguousarray(slot, np.int32)), int(len(chi_o) // 512),
                           _d(np.ascontiguousarray(chi_o, np.float64)),
                           _d(np.ascontiguousarray(udef_o, np.float64)),
                           _d(np.ascontiguousarray(kin, np.float64)), dt, lam, implicit, _d(F))
        return vel, F

    def pressure_rhs(self, vel, pres, dt, step, chi=None, slot=None, chi_o=None, udef_o=None):
        lhs = np.zeros(self.n)
        ns = 0 if chi_o is None else len(chi_o) // 512
        lib().orc_pressure_rhs(self._p, _d(np.ascontiguousarray(vel, np.float64)),
                               _d(np.ascontiguousarray(pres, np.float64)),
                               _d(None if chi is None else np.ascontiguousarray(chi, np.float64)),
                               _i(None if slot is None else np.ascontiguousarray(slot, np.int32)), ns,
                               _d(None if chi_o is None else np.ascontiguousarray(chi_o, np.float64)),
                               _d(None if udef_o is None else np.ascontiguousarray(udef_o, np.float64)),
                               dt, step, _d(lhs))
        return lhs

    def dissipation(self, vel, pres, chi, nu):
        """The 20 diagnostics of ComputeDissipation (circulation, linear impulse,
        linear momentum, angular impulse, angular momentum, pressure and viscous
        power, helicity, kinetic energy, enstrophy)."""
        out = np.zeros(20)
        lib().orc_dissipation(self._p, _d(np.ascontiguousarray(vel, np.float64)),
                              _d(np.ascontiguousarray(pres, np.float64)),
                              _d(None if chi is None else np.ascontiguousarray(chi, np.float64)), nu, _d(out))
        return out

    def create_obstacle(self, kind, centre, shape, quat=(1.0, 0.0, 0.0, 0.0)):
        """CreateObstacles' chi for a sphere (kind "sphere", shape = radius) or an
        ellipsoid (kind "ellipsoid", shape = semi-axes, quat = (w, x, y, z)).
        Returns dict(slot[nb], block_of_slot[ns], chi_o[ns*512], chi[nb*512],
        mass, com[3])."""
        nb = self.nb
        c = np.ascontiguousarray(centre, np.float64)
        sh = np.ascontiguousarray(np.atleast_1d(shape), np.float64)
        q = np.ascontiguousarray(quat, np.float64)
        slot = np.zeros(nb, np.int32)
        bos = np.zeros(nb, np.int32)
        chi_o = np.zeros(nb * 512)
        chi = np.zeros(nb * 512)
        mom = np.zeros(4)
        ns = lib().orc_create_obstacle(self._p, 0 if kind == "sphere" else 1, _d(c), _d(sh), _d(q), _i(slot),
                                       _i(bos), _d(chi_o), _d(chi), _d(mom))
        return dict(slot=slot, block_of_slot=bos[:ns].copy(), chi_o=chi_o[:ns * 512].copy(), chi=chi,
                    mass=mom[3], com=mom[:3] / mom[3] if mom[3] > 0 else np.zeros(3))

    def obstacle_surface(self, kind, centre, shape, block_of_slot, chi_o, quat=(1.0, 0.0, 0.0, 0.0)):
        """Surface points of the obstacle blocks: normals [3][ns][512] (zero off
        the surface), as ObstacleBlock::write records them (see oracle.cpp)."""
        bos = np.ascontiguousarray(block_of_slot, np.int32)
        ns = len(bos)
        nrm = np.zeros(3 * ns * 512)
        lib().orc_obstacle_surface(self._p, 0 if kind == "sphere" else 1,
                                   _d(np.ascontiguousarray(centre, np.float64)),
                                   _d(np.ascontiguousarray(np.atleast_1d(shape), np.float64)),
                                   _d(np.ascontiguousarray(quat, np.float64)), ns, _i(bos),
                                   _d(np.ascontiguousarray(chi_o, np.float64)), _d(nrm))
        return nrm

    def compute_forces(self, vel, pres, chi, block_of_slot, nrm, udef, nu, kin):
        """ComputeForces' 19 sums (surface, pressure and viscous force, torque,
        drag, thrust, Pout, PoutBnd, defPower, defPowerBnd, pLocom) and the
        number of surface points whose stencil left the same-level cells."""
        bos = np.ascontiguousarray(block_of_slot, np.int32)
        q = np.zeros(19)
        bad = lib().orc_compute_forces(self._p, _d(np.ascontiguousarray(vel, np.float64)),
                                       _d(np.ascontiguousarray(pres, np.float64)),
                                       _d(np.ascontiguousarray(chi, np.float64)), len(bos), _i(bos),
                                       _d(np.ascontiguousarray(nrm, np.float64)),
                                       _d(np.ascontiguousarray(udef, np.float64)), float(nu),
                                       _d(np.ascontiguousarray(kin, np.float64)), _d(q))
        return q, bad

    def adapt_indicator(self, vel, chi, level_max, level_max_vort, rtol, ctol):
        """Per-block refinement indicator of Simulation::adaptMesh (see oracle.cpp)."""
        out = np.zeros(self.nb)
        lib().orc_adapt_indicator(self._p, _d(np.ascontiguousarray(vel, np.float64)),
                                  _d(np.ascontiguousarray(chi, np.float64)), level_max, level_max_vort, rtol, ctol,
                                  _d(out))
        return out

    def adapt_leaves(self, indicator, rtol, ctol):
        """Leaves (level, i, j, k) after one adaptation, sorted."""
        cap = 8 * self.nb + 64
        out = np.zeros(4 * cap, np.int32)
        n = lib().orc_adapt_leaves(self._p, _d(np.ascontiguousarray(indicator, np.float64)), rtol, ctol, _i(out), cap)
        assert n <= cap
        return out[:4 * n].reshape(n, 4)

    def adapt_transfer(self, other, field, ncomp, vector_bc):
        """Moves a field of this mesh onto `other` (an oracle Mesh)."""
        f1 = np.zeros(ncomp * other.n)
        lib().orc_adapt_transfer(self._p, other._p, _d(np.ascontiguousarray(field, np.float64)), ncomp,
                                 1 if vector_bc else 0, _d(f1))
        return f1

    def grad_update(self, vel, pres, dt):
        vel = np.array(vel, np.float64)
        lib().orc_grad_update(self._p, _d(vel), _d(np.ascontiguousarray(pres, np.float64)), dt)
        return vel

    def pressure_project(self, vel, pres, dt, step, chi=None, slot=None, chi_o=None, udef_o=None,
                         mean_constraint=1, solver=0, tol=0.0, tol_rel=1e-12):
        vel = np.array(vel, np.float64)
        pres = np.array(pres, np.float64)
        if chi is None:
            chi = np.zeros(self.n)
        ns = 0 if chi_o is None else len(chi_o) // 512
        st = np.zeros(5)
        lhs = np.zeros(self.n)
        lib().orc_pressure_project(self._p, _d(vel), _d(pres), _d(np.ascontiguousarray(chi, np.float64)),
                                   _i(None if slot is None else np.ascontiguousarray(slot, np.int32)), ns,
                                   _d(None if chi_o is None else np.ascontiguousarray(chi_o, np.float64)),
                                   _d(None if udef_o is None else np.ascontiguousarray(udef_o, np.float64)),
                                   dt, step, mean_constraint, solver, tol, tol_rel, _d(st), _d(lhs))
        return vel, pres, dict(iterations=int(st[0]), restarts=int(st[1]), err_init=st[2], err_final=st[3],
                               converged=bool(st[4]), lhs=lhs)


def pinv():
    P = np.zeros(512 * 512)
    lib().orc_pinv(_d(P))
    return P


def dt(hmin, nu, cfl, umax, step, rampup):
    return lib().orc_dt(hmin, nu, cfl, umax, step, rampup)


def cnn_fwd_grad(params, x, target=None, C_=16, want_grad=True):
    """(out[n*512] float32, grad[nparam] or None, loss or None) of the CNN in FP64."""
    params = np.ascontiguousarray(params, np.float64)
    x = np.ascontiguousarray(x, np.float32)
    n = x.size // 1000
    out = np.zeros(n * 512, np.float32)
    grad = np.zeros(lib().orc_cnn_nparam(C_)) if (want_grad and target is not None) else None
    loss = np.zeros(1)
    t = None if target is None else np.ascontiguousarray(target, np.float32)
    lib().orc_cnn_fwd_grad(n, C_, _d(params), _f(x), _f(t), _f(out), _d(grad), _d(loss) if t is not None else None)
    return out, grad, (float(loss[0]) if t is not None else None)
