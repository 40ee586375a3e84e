"""cup3d_b200: B200-native time-step hot path of CubismUP_3D behind a C ABI.

Python is only a thin host layer over include/cup3d_b200.h (ctypes).  The
compute path is the sm_100a library cup3d_b200/libcup3d_b200.so; there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (ADV, BC, FIELD, FIELD_NCOMP, SOLVER, CupError, check, cup_config,
                   cup_solve_stats, dptr, iptr, lib)

__all__ = ["Context", "config", "CupError", "ADV", "BC", "SOLVER", "FIELD"]


def config(flags: str = "", **kw) -> cup_config:
    """Config with the reference's defaults, then `-key value` flags, then keywords."""
    cfg = cup_config()
    lib().cup_config_default(C.byref(cfg))
    if flags:
        check(lib().cup_config_parse(C.byref(cfg), flags.encode()))
    for k, v in kw.items():
        key = "lambda_" if k == "lambda" else k
        if key in ("bpd", "bc", "uinf"):
            arr = getattr(cfg, key)
            for i in range(3):
                arr[i] = v[i]
        else:
            setattr(cfg, key, v)
    return cfg


def _dev_ptr(t):
    """Raw device pointer of a torch CUDA tensor (float64, contiguous)."""
    import torch
    assert isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


class Context:
    """One simulation on one GPU (cup_ctx).  device=-1 gives a host-only
    context (mesh construction and tables only)."""

    def __init__(self, cfg: cup_config):
        self.cfg = cfg
        p = lib().cup_create(C.byref(cfg))
        if not p:
            raise CupError(-1, lib().cup_last_error(None).decode())
        self._p = C.c_void_p(p)

    def close(self):
        if getattr(self, "_p", None):
            lib().cup_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- mesh -------------------------------------------------------------
    def set_mesh(self, level, index):
        level = np.ascontiguousarray(level, dtype=np.int32)
        index = np.ascontiguousarray(index, dtype=np.int32).reshape(-1)
        check(lib().cup_set_mesh(self._p, len(level), iptr(level), iptr(index)), self._p)

    def set_mesh_uniform(self):
        check(lib().cup_set_mesh_uniform(self._p), self._p)

    def set_mesh_sphere_wake(self, center, radius, flow_dir=-1, near_radius=0.3, wake_len=1.0,
                             wake_radius=0.3):
        c = np.ascontiguousarray(center, dtype=np.float64)
        check(lib().cup_set_mesh_sphere_wake(self._p, dptr(c), radius, flow_dir, near_radius,
                                             wake_len, wake_radius), self._p)

    def set_mesh_random(self, seed, prob):
        check(lib().cup_set_mesh_random(self._p, seed, prob), self._p)

    @property
    def nb(self) -> int:
        return lib().cup_num_blocks(self._p)

    def blocks(self):
        nb = self.nb
        level = np.zeros(nb, np.int32)
        index = np.zeros(3 * nb, np.int32)
        h = np.zeros(nb, np.float64)
        check(lib().cup_get_blocks(self._p, iptr(level), iptr(index), dptr(h)), self._p)
        return level, index.reshape(nb, 3), h

    def cell_centres(self):
        """Physical cell centres (nb*512, 3) and cell sizes (nb*512,) in device block order."""
        level, index, h = self.blocks()
        ix = np.arange(512) % 8
        iy = (np.arange(512) // 8) % 8
        iz = np.arange(512) // 64
        xyz = np.zeros((len(level), 512, 3))
        for d, i in enumerate((ix, iy, iz)):
            xyz[:, :, d] = (index[:, d:d + 1] * 8 + i[None, :] + 0.5) * h[:, None]
        return xyz.reshape(-1, 3), np.repeat(h, 512)

    def faces(self):
        nb = self.nb
        kinds = np.zeros(6 * nb, np.int32)
        nbrs = np.zeros(24 * nb, np.int32)
        check(lib().cup_get_faces(self._p, iptr(kinds), iptr(nbrs)), self._p)
        return kinds.reshape(nb, 6), nbrs.reshape(nb, 6, 4)

    # ---- fields -----------------------------------------------------------
    def upload(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        assert a.size == FIELD_NCOMP[name] * self.nb * 512
        check(lib().cup_upload_field(self._p, FIELD[name], dptr(a)), self._p)

    def download(self, name):
        a = np.zeros(FIELD_NCOMP[name] * self.nb * 512, np.float64)
        check(lib().cup_download_field(self._p, FIELD[name], dptr(a)), self._p)
        return a

    def upload_blocks(self, name, level, index, blocks):
        """Upload from the reference's block storage: blocks[k] holds the 512
        cells ([iz][iy][ix]) of block (level[k], index[k]), components interleaved."""
        arrs = [np.ascontiguousarray(b, dtype=np.float64).reshape(-1) for b in blocks]
        lv = np.ascontiguousarray(level, np.int32)
        ix = np.ascontiguousarray(np.asarray(index).reshape(-1), np.int32)
        ptrs = (_lib._D * len(arrs))(*[dptr(a) for a in arrs])
        check(lib().cup_upload_field_blocks(self._p, FIELD[name], len(arrs), iptr(lv), iptr(ix), ptrs), self._p)

    def download_blocks(self, name, level, index):
        """Download into the reference's block storage (one array per block)."""
        lv = np.ascontiguousarray(level, np.int32)
        ix = np.ascontiguousarray(np.asarray(index).reshape(-1), np.int32)
        arrs = [np.zeros(512 * FIELD_NCOMP[name], np.float64) for _ in range(len(lv))]
        ptrs = (_lib._D * len(arrs))(*[dptr(a) for a in arrs])
        check(lib().cup_download_field_blocks(self._p, FIELD[name], len(arrs), iptr(lv), iptr(ix), ptrs), self._p)
        return arrs

    def field_ptr(self, name) -> int:
        return lib().cup_field_device_ptr(self._p, FIELD[name])

    # ---- raw device operators (torch CUDA float64 tensors) ----------------
    def poisson_apply(self, x, y, mean_mode=-1):
        check(lib().cup_poisson_apply_dev(self._p, _dev_ptr(x), _dev_ptr(y), mean_mode), self._p)

    def block_inverse(self, x, y):
        check(lib().cup_block_inverse_dev(self._p, _dev_ptr(x), _dev_ptr(y)), self._p)

    def poisson_solve_dev(self, b, x):
        st = cup_solve_stats()
        rc = check(lib().cup_poisson_solve_dev(self._p, _dev_ptr(b), _dev_ptr(x), C.byref(st)), self._p)
        return rc, st.as_dict()

    def poisson_solve(self):
        """PoissonSolverBase::solve(): RHS in 'lhs', guess/result in 'pres'."""
        st = cup_solve_stats()
        rc = check(lib().cup_poisson_solve(self._p, C.byref(st)), self._p)
        return rc, st.as_dict()

    # ---- obstacles ----------------------------------------------------------
    def obstacle_sphere(self, center, radius, vel=(0, 0, 0), omega=(0, 0, 0), on_device=False):
        """Sphere body; on_device: created by kernels (cup_obstacle_sphere_dev)."""
        c, v, o = (np.ascontiguousarray(a, dtype=np.float64) for a in (center, vel, omega))
        fn = lib().cup_obstacle_sphere_dev if on_device else lib().cup_obstacle_sphere
        check(fn(self._p, dptr(c), radius, dptr(v), dptr(o)), self._p)

    def obstacle_ellipsoid(self, center, axes, quat, vel=(0, 0, 0), omega=(0, 0, 0), on_device=False):
        """Ellipsoid body; on_device: created by kernels (cup_obstacle_ellipsoid_dev)."""
        c, a, q, v, o = (np.ascontiguousarray(x, dtype=np.float64) for x in (center, axes, quat, vel, omega))
        fn = lib().cup_obstacle_ellipsoid_dev if on_device else lib().cup_obstacle_ellipsoid
        check(fn(self._p, dptr(c), dptr(a), dptr(q), dptr(v), dptr(o)), self._p)

    def obstacle_free(self, trans=(1, 1, 1), rot=(1, 1, 1)):
        """Free degrees of freedom of the body (cup_obstacle_free)."""
        t, r = (np.ascontiguousarray(x, np.int32) for x in (trans, rot))
        check(lib().cup_obstacle_free(self._p, iptr(t), iptr(r)), self._p)

    def obstacle_fix_frame(self, fix=(1, 0, 0)):
        """The frame of reference follows the body along these axes (cup_obstacle_fix_frame)."""
        f = np.ascontiguousarray(fix, np.int32)
        check(lib().cup_obstacle_fix_frame(self._p, iptr(f)), self._p)

    def uinf(self):
        """The frame velocity in use (cup_get_uinf)."""
        u = np.zeros(3)
        check(lib().cup_get_uinf(self._p, dptr(u)), self._p)
        return u

    def update_obstacles(self, dt):
        """UpdateObstacles (cup_update_obstacles): dict of the body's velocity,
        angular velocity, force and torque."""
        out = np.zeros(12)
        check(lib().cup_update_obstacles(self._p, dt, dptr(out)), self._p)
        return {"vel": out[0:3], "omega": out[3:6], "force": out[6:9], "torque": out[9:12]}

    def dissipation(self):
        """ComputeDissipation's 20 diagnostics of the current state (cup_compute_dissipation)."""
        out = np.zeros(20)
        check(lib().cup_compute_dissipation(self._p, dptr(out)), self._p)
        return out

    def write_restart(self, directory, step, time):
        """Restart files of step `step` in `directory` (cup_write_restart)."""
        check(lib().cup_write_restart(self._p, str(directory).encode(), step, time), self._p)

    def read_restart(self, directory, step):
        """Restores the state saved at step `step` (cup_read_restart); returns the saved time."""
        t = np.zeros(1)
        check(lib().cup_read_restart(self._p, str(directory).encode(), step, dptr(t)), self._p)
        return float(t[0])

    def set_obstacle(self, blocks, chi, udef, kin):
        blocks = np.ascontiguousarray(blocks, np.int32)
        chi, udef, kin = (np.ascontiguousarray(x, np.float64) for x in (chi, udef, kin))
        check(lib().cup_set_obstacle(self._p, len(blocks), iptr(blocks), dptr(chi), dptr(udef), dptr(kin)), self._p)

    def get_obstacle(self):
        """(slot_of_block[nb], chi[nslots*512], udef[3*nslots*512], kin[9])"""
        ns = check(lib().cup_get_obstacle(self._p, None, None, None, None), self._p)
        blocks = np.zeros(ns, np.int32)
        chi = np.zeros(ns * 512)
        udef = np.zeros(3 * ns * 512)
        kin = np.zeros(9)
        check(lib().cup_get_obstacle(self._p, iptr(blocks), dptr(chi), dptr(udef), dptr(kin)), self._p)
        slot = -np.ones(self.nb, np.int32)
        slot[blocks] = np.arange(ns, dtype=np.int32)
        return slot, chi, udef, kin

    # ---- time-step operators -------------------------------------------------
    def max_u(self):
        out = C.c_double()
        check(lib().cup_max_u(self._p, C.byref(out)), self._p)
        return out.value

    def compute_dt(self, step):
        out = C.c_double()
        check(lib().cup_compute_dt(self._p, step, C.byref(out)), self._p)
        return out.value

    def advect_diffuse(self, dt):
        check(lib().cup_advect_diffuse(self._p, dt), self._p)

    def penalize(self, dt):
        f = np.zeros(6)
        check(lib().cup_penalize(self._p, dt, dptr(f)), self._p)
        return f

    def pressure_project(self, dt, step):
        st = cup_solve_stats()
        rc = check(lib().cup_pressure_project(self._p, dt, step, C.byref(st)), self._p)
        return rc, st.as_dict()

    def step(self, step, dt=0.0):
        used = C.c_double()
        st = cup_solve_stats()
        rc = check(lib().cup_step(self._p, step, dt, C.byref(used), C.byref(st)), self._p)
        return used.value, rc, st.as_dict()

    def autotune(self):
        """Picks launch grids by timing (cup_autotune): ({kernel: grid}, {kernel: ms})."""
        ch = (C.c_int32 * 4)()
        ms = (C.c_float * 4)()
        check(lib().cup_autotune(self._p, ch, ms), self._p)
        names = ("advect", "pressure_rhs", "grad_update", "solver")
        return dict(zip(names, list(ch))), dict(zip(names, list(ms)))

    # ---- profiling ----------------------------------------------------------
    def profile(self, enable=True):
        check(lib().cup_profile(self._p, int(enable)), self._p)

    def profile_read(self):
        """{phase: (launches, milliseconds)} accumulated since profile(True)."""
        import json
        buf = C.create_string_buffer(1 << 16)
        check(lib().cup_profile_read(self._p, buf, len(buf)), self._p)
        return {k: (int(v[0]), float(v[1])) for k, v in json.loads(buf.value.decode()).items()}

    # ---- solver settings ------------------------------------------------------
    def set_poisson(self, solver="b200", tol_abs=1e-6, tol_rel=1e-4, max_iter=1000):
        check(lib().cup_set_poisson(self._p, SOLVER[solver], tol_abs, tol_rel, max_iter), self._p)

    def adapt_indicator(self):
        """Each block's refinement indicator (cup_adapt_indicator)."""
        out = np.zeros(self.nb)
        check(lib().cup_adapt_indicator(self._p, dptr(out)), self._p)
        return out

    def adapt_mesh(self):
        """One mesh adaptation (Simulation::adaptMesh); True when the mesh changed."""
        ch = C.c_int32(0)
        check(lib().cup_adapt_mesh(self._p, C.byref(ch)), self._p)
        return bool(ch.value)

    def cnn_holdout(self, ntest):
        check(lib().cup_cnn_holdout(self._p, int(ntest)), self._p)

    def cnn_eval(self):
        """Held-out mean squared error relative to the held-out mean square target."""
        out = C.c_float(0)
        check(lib().cup_cnn_eval(self._p, C.byref(out)), self._p)
        return out.value

    def coarse_matrix(self):
        """(A_c (nb, nb), colours) of the two-level solvers' coarse space."""
        nb = self.nb
        out = np.zeros(nb * nb)
        col = C.c_int32(0)
        check(lib().cup_coarse_matrix(self._p, dptr(out), C.byref(col)), self._p)
        return out.reshape(nb, nb), col.value

    def coarse_apply(self, r, z):
        """z = P A_c^-1 P^T r on torch CUDA float64 tensors."""
        check(lib().cup_coarse_apply_dev(self._p, _dev_ptr(r), _dev_ptr(z)), self._p)

    def dense_inverse(self, a, last=-1):
        """a <- a^-1 in place (torch CUDA float64, n x n, row-major), by the
        coarse space's device inverse; True when the pivoted form ran."""
        n = int(a.shape[0])
        assert a.dtype.is_floating_point and a.element_size() == 8 and a.is_contiguous() and a.shape == (n, n)
        piv = C.c_int32(0)
        check(lib().cup_dense_inverse_dev(self._p, _dev_ptr(a), n, int(last), C.byref(piv)), self._p)
        return bool(piv.value)

    def set_barrier_limit(self, cycles):
        """Wait limit of the persistent solvers' grid barriers (0: default)."""
        check(lib().cup_set_barrier_limit(self._p, int(cycles)), self._p)

    def pressure_rhs(self, dt, step):
        """Opens a split projection: the Poisson right-hand side into the 'lhs'
        field; 'pres' is then the (zero) pressure increment that poisson_solve
        solves for, until pressure_finish."""
        check(lib().cup_pressure_rhs(self._p, dt, step), self._p)

    def pressure_finish(self, dt, step):
        """Closes a split projection: zero mean, p += p_old, gradient update."""
        check(lib().cup_pressure_finish(self._p, dt, step), self._p)

    # ---- learned preconditioner -------------------------------------------------
    @staticmethod
    def cnn_num_params():
        return lib().cup_cnn_num_params()

    def cnn_init(self, seed=0):
        check(lib().cup_cnn_init(self._p, seed), self._p)

    def cnn_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.cnn_num_params()
        check(lib().cup_cnn_set_params(self._p, p.ctypes.data_as(C.POINTER(C.c_float))), self._p)

    def cnn_get_params(self):
        p = np.zeros(self.cnn_num_params(), np.float32)
        check(lib().cup_cnn_get_params(self._p, p.ctypes.data_as(C.POINTER(C.c_float))), self._p)
        return p

    def cnn_dataset_reserve(self, capacity):
        check(lib().cup_cnn_dataset_reserve(self._p, capacity), self._p)

    def cnn_dataset_add(self, r, e=None):
        """One sample per block from the device residual r of a solver iterate
        (target: the one-cell-overlap local solve's correction; e, the
        iterate's error, is not used)."""
        check(lib().cup_cnn_dataset_add(self._p, _dev_ptr(r), _dev_ptr(e) if e is not None else None), self._p)

    def cnn_dataset_size(self):
        return lib().cup_cnn_dataset_size(self._p)

    def cnn_train(self, steps, batch=64, lr=1e-3, seed=0):
        losses = np.zeros(max(steps, 1), np.float32)
        check(lib().cup_cnn_train(self._p, steps, batch, lr, seed, losses.ctypes.data_as(C.POINTER(C.c_float))),
              self._p)
        return losses[:steps]

    def cnn_forward(self, x, n):
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros(n * 512, np.float32)
        fp = C.POINTER(C.c_float)
        check(lib().cup_cnn_forward_host(self._p, x.ctypes.data_as(fp), out.ctypes.data_as(fp), n), self._p)
        return out

    def cnn_forward_noalloc(self, x, n):
        """cnn_forward without device allocation (at most 64 samples per call)."""
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros(n * 512, np.float32)
        fp = C.POINTER(C.c_float)
        check(lib().cup_cnn_forward_host_noalloc(self._p, x.ctypes.data_as(fp), out.ctypes.data_as(fp), n), self._p)
        return out

    def cnn_grad(self, x, target, n):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        g = np.zeros(self.cnn_num_params(), np.float32)
        loss = np.zeros(1, np.float32)
        fp = C.POINTER(C.c_float)
        check(lib().cup_cnn_grad_host(self._p, x.ctypes.data_as(fp), t.ctypes.data_as(fp), n, g.ctypes.data_as(fp),
                                      loss.ctypes.data_as(fp)), self._p)
        return g, float(loss[0])

    def cnn_precond(self, r, z):
        check(lib().cup_cnn_precond_dev(self._p, _dev_ptr(r), _dev_ptr(z)), self._p)

    def cnn_map_apply(self, r, z):
        """z = block inverse + folded network on r, the solver's path."""
        check(lib().cup_cnn_map_apply_dev(self._p, _dev_ptr(r), _dev_ptr(z)), self._p)

    FORCE_KEYS = ("surfForce", "presForce", "viscForce", "surfTorque")
    FORCE_SCALARS = ("drag", "thrust", "Pout", "PoutBnd", "defPower", "defPowerBnd", "pLocom", "Pthrust", "Pdrag",
                     "EffPDef", "EffPDefBnd")

    def compute_forces(self):
        """ComputeForces on the current velocity and pressure: dict of the
        surface force, its pressure and viscous parts, the torque (arrays of 3)
        and the scalar quantities of Obstacle::computeForces."""
        out = np.zeros(23)
        check(lib().cup_compute_forces(self._p, dptr(out)), self._p)
        res = {k: out[3 * i:3 * i + 3].copy() for i, k in enumerate(self.FORCE_KEYS)}
        res.update({k: float(out[12 + i]) for i, k in enumerate(self.FORCE_SCALARS)})
        res["raw"] = out
        return res

    def schwarz_apply(self, r, z):
        """z = block inverse + the one-cell-overlap local solve's correction on r."""
        check(lib().cup_schwarz_apply_dev(self._p, _dev_ptr(r), _dev_ptr(z)), self._p)
class Batch(Context):
    """Independent cases in one context (cup_batch_create): the cases' meshes
    concatenated in case order; their Poisson solves run in one device
    launch, each case with its own BiCGSTAB."""

    def __init__(self, cases):
        cases = list(cases)
        arr = (C.c_void_p * len(cases))(*[c._p.value for c in cases])
        p = lib().cup_batch_create(len(cases), arr)
        if not p:
            raise CupError(-1, lib().cup_last_error(None).decode())
        self.cfg = cases[0].cfg
        self._p = C.c_void_p(p)
        self.ncase = int(lib().cup_batch_num_cases(self._p))

    def case_blocks(self, k):
        """(first block, number of blocks) of case k."""
        first, n = C.c_int32(), C.c_int32()
        check(lib().cup_batch_case_blocks(self._p, k, C.byref(first), C.byref(n)), self._p)
        return first.value, n.value

    def step(self, step, dt=None):
        """One time step of every case: (rc, dt per case, force/torque (ncase, 6),
        [stats per case]).  dt: per-case time steps, None for each case's CFL."""
        dt_in = None if dt is None else np.ascontiguousarray(dt, np.float64)
        dt_used = np.zeros(self.ncase)
        force = np.zeros((self.ncase, 6))
        st = (cup_solve_stats * self.ncase)()
        rc = check(lib().cup_batch_step(self._p, step, None if dt_in is None else dptr(dt_in), dptr(dt_used),
                                        dptr(force), st), self._p)
        return rc, dt_used, force, [s.as_dict() for s in st]

    def case_field(self, name, k):
        """Case k's part of a downloaded field, (ncomp, nblocks*512)."""
        first, n = self.case_blocks(k)
        f = self.download(name).reshape(FIELD_NCOMP[name], -1)
        return f[:, first * 512:(first + n) * 512]

    def poisson_solve_dev(self, b, x):
        """One BiCGSTAB per case in one launch: (rc, [stats per case])."""
        st = (cup_solve_stats * self.ncase)()
        rc = check(lib().cup_batch_poisson_solve_dev(self._p, _dev_ptr(b), _dev_ptr(x), st), self._p)
        return rc, [s.as_dict() for s in st]


