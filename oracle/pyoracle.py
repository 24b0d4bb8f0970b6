"""ctypes binding of the FP64 OpenMP oracle (oracle/aw_oracle.cpp).

Test infrastructure only: imported by tests/, by ``__graft_entry__.smoke()`` and by the
CPU-baseline legs of ``bench.py``.  The product library never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_SRC = os.path.join(_HERE, "aw_oracle.cpp")

CXXFLAGS = ["-O3", "-march=x86-64-v2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-Wall"]


def build(force: bool = False) -> str:
    """Compile the oracle into oracle/liboracle.so (g++ + OpenMP)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(_SRC):
        subprocess.check_call(["g++", *CXXFLAGS, "-o", _SO, _SRC])
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_SO)
        P = C.c_void_p
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
        u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
        L.oc_morton3d.restype = C.c_uint32
        L.oc_morton3d.argtypes = [C.c_uint32] * 3
        L.oc_block_layout.argtypes = [C.c_int, C.c_int, u32p]
        L.oc_num_threads.restype = C.c_int
        L.oc_set_threads.argtypes = [C.c_int]
        L.oc_levels_from_particles.argtypes = [i32p, C.c_float, f32p, C.c_int, C.c_int, f32p, C.c_int64, i32p, u32p]
        L.oc_enforce_grading.argtypes = [i32p, C.c_int, u32p, i32p]
        L.oc_create.restype = P
        L.oc_create.argtypes = [i32p, C.c_float, f32p, C.c_int, C.c_int, u32p]
        L.oc_destroy.argtypes = [P]
        L.oc_set_params.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                    C.c_double, C.c_double, C.c_double]
        L.oc_offsets.argtypes = [P, C.c_int, C.c_int, u32p, u32p]
        L.oc_galerkin_ref.argtypes = [P, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.oc_build.restype = C.c_int
        L.oc_build.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.oc_num_levels.restype = C.c_int
        L.oc_num_levels.argtypes = [P]
        L.oc_level_info.argtypes = [P, C.c_int, i64p]
        L.oc_get.argtypes = [P, C.c_int, C.c_int, f64p]
        L.oc_set.argtypes = [P, C.c_int, C.c_int, f64p]
        for fn in ("oc_smooth",):
            getattr(L, fn).argtypes = [P, C.c_int, C.c_int]
        for fn in ("oc_residual", "oc_restrict", "oc_prolong"):
            getattr(L, fn).argtypes = [P, C.c_int]
        L.oc_vcycle.argtypes = [P]
        L.oc_coarsest.argtypes = [P]
        L.oc_solve.restype = C.c_int
        L.oc_solve.argtypes = [P, f64p, f64p, C.c_double, C.c_int, C.c_void_p]
        L.oc_apply.argtypes = [P, C.c_int, f64p, f64p]
        L.oc_particle_keys.argtypes = [P, f32p, C.c_int64, u32p, i64p]
        L.oc_p2g.argtypes = [P, f32p, f32p, C.c_int64, f64p, f64p, f64p, f64p, f64p, f64p, u32p]
        L.oc_p2g_phase.argtypes = [P, f32p, f32p, f32p, C.c_int64] + [f64p] * 9 + [u32p]
        L.oc_beta_sync.argtypes = [P, f64p, f64p, f64p]
        L.oc_face_sync.argtypes = [P, f64p, f64p, f64p]
        L.oc_wall_bc.argtypes = [P, f64p, f64p, f64p]
        L.oc_divergence.argtypes = [P, f64p, f64p, f64p, u8p, C.c_double, f64p]
        L.oc_gradient_update.argtypes = [P, f64p, C.c_double, f64p, f64p, f64p]
        L.oc_g2p.argtypes = [P, f32p, C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_double, f32p, f64p]
        L.oc_sample.argtypes = [P, f64p, C.c_int64, C.POINTER(C.c_void_p), f64p]
        L.oc_advect.argtypes = [P, C.POINTER(C.c_void_p), C.c_double, f64p, C.c_int64, f64p]
        # FP64 particle state and the adjoint (VJP) of the FLIP step
        L.oc_p2g64.argtypes = [P, f64p, f64p, C.c_int64, f64p, f64p, f64p, f64p, f64p, f64p, u32p]
        L.oc_g2p64.argtypes = [P, f64p, C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_double, f64p,
                               f64p]
        L.oc_sample_stencil.argtypes = [P, f64p, C.c_int64, C.POINTER(C.c_void_p), f64p]
        L.oc_sample_vjp.argtypes = [P, f64p, C.c_int64, C.POINTER(C.c_void_p), f64p, C.POINTER(C.c_void_p),
                                    C.c_void_p]
        L.oc_g2p_vjp.argtypes = [P, f64p, C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_double, f64p,
                                 f64p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.oc_advect_vjp.argtypes = [P, C.POINTER(C.c_void_p), C.c_double, f64p, C.c_int64, f64p, C.POINTER(C.c_void_p)]
        L.oc_p2g_vjp.argtypes = [P, f64p, f64p, C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                 C.POINTER(C.c_void_p), f64p, f64p]
        L.oc_face_sync_vjp.argtypes = [P, f64p, f64p, f64p]
        L.oc_set_coarse_all.argtypes = [P, C.c_int]
        L.oc_divergence_vjp.argtypes = [P, f64p, u8p, C.c_double, f64p, f64p, f64p]
        L.oc_gradient_vjp.argtypes = [P, C.c_double, f64p, f64p, f64p, f64p]
        _lib = L
    return _lib


def _ptrs(arrs):
    return (C.c_void_p * 3)(*[a.ctypes.data for a in arrs])


def morton3d(x, y, z):
    return lib().oc_morton3d(x, y, z)


def block_layout(R0, level):
    out = np.zeros(6, np.uint32)
    lib().oc_block_layout(R0, level, out)
    return out


def num_threads():
    return lib().oc_num_threads()


def set_threads(n):
    lib().oc_set_threads(int(n))


def levels_from_particles(dims, bs, dmin, R0, L, pos, thresholds):
    dims = np.ascontiguousarray(dims, np.int32)
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    th = np.ascontiguousarray(list(thresholds) + [0], np.int32)
    out = np.zeros(int(np.prod(dims)), np.uint32)
    lib().oc_levels_from_particles(dims, float(bs), np.ascontiguousarray(dmin, np.float32), R0, L, pos,
                                   pos.shape[0], th, out)
    return out


def enforce_grading(dims, L, levels):
    lv = np.ascontiguousarray(levels, np.uint32).copy()
    passes = np.zeros(1, np.int32)
    lib().oc_enforce_grading(np.ascontiguousarray(dims, np.int32), L, lv, passes)
    return lv, int(passes[0])


class Oracle:
    """FP64 restatement of one MSBG grid + its multigrid hierarchy."""

    def __init__(self, dims, bs, dmin, R0, L, levels):
        self.dims = np.ascontiguousarray(dims, np.int32)
        self.bs, self.R0, self.L = float(bs), int(R0), int(L)
        self.dmin = np.ascontiguousarray(dmin, np.float32)
        self.levels = np.ascontiguousarray(levels, np.uint32)
        self.nb = int(np.prod(self.dims))
        self.h = lib().oc_create(self.dims, self.bs, self.dmin, self.R0, self.L, self.levels)
        off, tot = self.offsets(0, True)
        self.off0, self.tot0 = off, tot

    def __del__(self):
        try:
            if self.h:
                lib().oc_destroy(self.h)
        except Exception:
            pass

    def set_params(self, mode=0, pre=2, post=2, coarsest_iters=50, block_iters=None, dense_sweeps=2,
                   omega=None, target=0.33, theta=None, lam=1.0):
        """Defaults follow the library's: FV mode (block_iters 2, omega 1.35 as a float32, every
        block active: theta -1); reference mode (Smoother.cuh:9-11,286: block_iters 10, omega
        0.85714, theta 1e-4)."""
        ref = mode == 1
        block_iters = (10 if ref else 2) if block_iters is None else block_iters
        omega = (0.85714 if ref else float(np.float32(1.35))) if omega is None else omega
        theta = (1e-4 if ref else -1.0) if theta is None else theta
        lib().oc_set_params(self.h, mode, pre, post, coarsest_iters, block_iters, dense_sweeps, omega, target,
                            theta, lam)

    def offsets(self, m, vanish=True):
        out = np.zeros(4 * self.nb, np.uint32)
        tot = np.zeros(4, np.uint32)
        lib().oc_offsets(self.h, m, int(vanish), out, tot)
        return out.reshape(4, self.nb), tot

    def galerkin_ref(self, dest, fine):
        _, totc = self.offsets(dest, True)
        fine = [np.ascontiguousarray(f, np.float32) for f in fine]
        coarse = [np.zeros(int(totc[1 + a]), np.float32) for a in range(3)]
        lib().oc_galerkin_ref(self.h, dest, _ptrs(fine), _ptrs(coarse))
        return coarse

    def build(self, bbar=None, fluid=None, mg_levels=0):
        keep = []

        def p(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a.ctypes.data

        bb = bbar if bbar is not None else (None, None, None)
        n = lib().oc_build(self.h, p(bb[0], np.float64), p(bb[1], np.float64), p(bb[2], np.float64),
                           p(fluid, np.uint8), mg_levels)
        return n

    def num_levels(self):
        return lib().oc_num_levels(self.h)

    def level_info(self, m):
        out = np.zeros(8, np.int64)
        lib().oc_level_info(self.h, m, out)
        return out

    def _size(self, m, which):
        info = self.level_info(m)
        if which in (0, 1, 2, 6):
            return int(info[4])
        return int(info[5 + which - 3])

    def get(self, m, which):
        out = np.zeros(self._size(m, which), np.float64)
        lib().oc_get(self.h, m, which, out)
        return out

    def set(self, m, which, arr):
        lib().oc_set(self.h, m, which, np.ascontiguousarray(arr, np.float64))

    def smooth(self, m, iters):
        lib().oc_smooth(self.h, m, iters)

    def residual(self, m):
        lib().oc_residual(self.h, m)

    def restrict(self, m):
        lib().oc_restrict(self.h, m)

    def prolong(self, m):
        lib().oc_prolong(self.h, m)

    def vcycle(self):
        lib().oc_vcycle(self.h)

    def coarsest(self):
        lib().oc_coarsest(self.h)

    def solve(self, b, tol=1e-6, max_cycles=100, p0=None, method="dc"):
        """FP64 solve of A p = b on level 0.  method "dc": V-cycle defect correction (oc_solve);
        "pcg": conjugate gradients preconditioned by the same V-cycle (the library's mixed-precision
        outer loop)."""
        n = int(self.level_info(0)[4])
        p = np.zeros(n) if p0 is None else np.ascontiguousarray(p0, np.float64).copy()
        b = np.ascontiguousarray(b, np.float64)
        if method == "pcg":
            return self._pcg(b, p, tol, max_cycles)
        hist = np.zeros(max_cycles + 1)
        it = lib().oc_solve(self.h, p, b, tol, max_cycles, hist.ctypes.data)
        return p, hist[: it + 1]

    def _pcg(self, b, p, tol, max_cycles):
        fl = self.get(0, 6) != 0
        n = p.size

        def V(r):
            self.set(0, 1, r)
            self.set(0, 0, np.zeros(n))
            self.vcycle()
            return self.get(0, 0)

        bn = np.linalg.norm(b * fl) or 1.0
        r = (b - self.apply(0, p)) * fl
        hist = [np.linalg.norm(r) / bn]
        z = V(r) * fl
        d = z.copy()
        rho = r @ z
        while hist[-1] >= tol and len(hist) <= max_cycles:
            q = self.apply(0, d) * fl
            alpha = rho / (d @ q)
            p += alpha * d
            r -= alpha * q
            hist.append(np.linalg.norm(r) / bn)
            z = V(r) * fl
            rn = r @ z
            d = z + (rn / rho) * d
            rho = rn
        return p, np.array(hist)

    def apply(self, m, x):
        y = np.zeros_like(np.ascontiguousarray(x, np.float64))
        lib().oc_apply(self.h, m, np.ascontiguousarray(x, np.float64), y)
        return y

    # ---- particles --------------------------------------------------------------------------
    def particle_keys(self, pos):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        n = pos.shape[0]
        keys = np.zeros(n, np.uint32)
        perm = np.zeros(n, np.int64)
        lib().oc_particle_keys(self.h, pos, n, keys, perm)
        return keys, perm

    def p2g(self, pos, vel):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        t = self.tot0
        u = [np.zeros(int(t[1 + a])) for a in range(3)]
        m = [np.zeros(int(t[1 + a])) for a in range(3)]
        cnt = np.zeros(int(t[0]), np.uint32)
        lib().oc_p2g(self.h, pos, vel, pos.shape[0], u[0], u[1], u[2], m[0], m[1], m[2], cnt)
        return u, m, cnt

    def p2g_phase(self, pos, vel, phase):
        """p2g plus the face phase sum w phase / sum w (0 where the mass is <= 1e-6)."""
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        phase = np.ascontiguousarray(phase, np.float32).reshape(-1)
        t = self.tot0
        u = [np.zeros(int(t[1 + a])) for a in range(3)]
        m = [np.zeros(int(t[1 + a])) for a in range(3)]
        phi = [np.zeros(int(t[1 + a])) for a in range(3)]
        cnt = np.zeros(int(t[0]), np.uint32)
        lib().oc_p2g_phase(self.h, pos, vel, phase, pos.shape[0], u[0], u[1], u[2], m[0], m[1], m[2], phi[0], phi[1],
                           phi[2], cnt)
        return u, m, cnt, phi

    def beta_sync(self, beta):
        """T-junction coefficients: the coarse face and its 4 fine faces all take the fine mean."""
        beta = [np.ascontiguousarray(x, np.float64).copy() for x in beta]
        lib().oc_beta_sync(self.h, *beta)
        return beta

    def phase_beta(self, phi, rho0, rho1):
        """beta = 1 / ((1 - phi) rho0 + phi rho1), then the T-junction sync."""
        return self.beta_sync([1.0 / ((1.0 - f) * rho0 + f * rho1) for f in phi])

    def face_sync(self, u):
        u = [np.ascontiguousarray(x, np.float64).copy() for x in u]
        lib().oc_face_sync(self.h, *u)
        return u

    def wall_bc(self, u):
        u = [np.ascontiguousarray(x, np.float64).copy() for x in u]
        lib().oc_wall_bc(self.h, *u)
        return u

    def divergence(self, u, fluid, dt):
        b = np.zeros(int(self.tot0[0]))
        u = [np.ascontiguousarray(x, np.float64) for x in u]
        lib().oc_divergence(self.h, u[0], u[1], u[2], np.ascontiguousarray(fluid, np.uint8), 1.0 / dt, b)
        return b

    def gradient_update(self, p, dt, u):
        u = [np.ascontiguousarray(x, np.float64).copy() for x in u]
        lib().oc_gradient_update(self.h, np.ascontiguousarray(p, np.float64), dt, *u)
        return u

    def g2p(self, pos, un, uo, alpha, vel):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        un = [np.ascontiguousarray(x, np.float64) for x in un]
        uo = [np.ascontiguousarray(x, np.float64) for x in uo]
        out = np.zeros((pos.shape[0], 3))
        lib().oc_g2p(self.h, pos, pos.shape[0], _ptrs(un), _ptrs(uo), alpha,
                     np.ascontiguousarray(vel, np.float32).reshape(-1, 3), out)
        return out

    def sample(self, X, u):
        X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
        u = [np.ascontiguousarray(x, np.float64) for x in u]
        out = np.zeros_like(X)
        lib().oc_sample(self.h, X, X.shape[0], _ptrs(u), out)
        return out

    # ---- FP64 particle state and VJPs (the differentiable rollout) ------------------------------
    def _faces(self):
        t = self.tot0
        return [np.zeros(int(t[1 + a])) for a in range(3)]

    def p2g64(self, pos, vel):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, np.float64).reshape(-1, 3)
        u, m = self._faces(), self._faces()
        cnt = np.zeros(int(self.tot0[0]), np.uint32)
        lib().oc_p2g64(self.h, pos, vel, pos.shape[0], u[0], u[1], u[2], m[0], m[1], m[2], cnt)
        return u, m, cnt

    def g2p64(self, pos, un, uo, alpha, vel):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        un = [np.ascontiguousarray(x, np.float64) for x in un]
        uo = [np.ascontiguousarray(x, np.float64) for x in uo]
        out = np.zeros_like(pos)
        lib().oc_g2p64(self.h, pos, pos.shape[0], _ptrs(un), _ptrs(uo), alpha,
                       np.ascontiguousarray(vel, np.float64).reshape(-1, 3), out)
        return out

    def sample_vjp(self, X, u, ybar, ubar, Xbar=None):
        X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
        u = [np.ascontiguousarray(x, np.float64) for x in u]
        lib().oc_sample_vjp(self.h, X, X.shape[0], _ptrs(u), np.ascontiguousarray(ybar, np.float64).reshape(-1, 3),
                            _ptrs(ubar), None if Xbar is None else Xbar.ctypes.data)

    def g2p_vjp(self, X, un, uo, alpha, vbar, Xbar, unbar, uobar):
        X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
        un = [np.ascontiguousarray(x, np.float64) for x in un]
        uo = [np.ascontiguousarray(x, np.float64) for x in uo]
        lib().oc_g2p_vjp(self.h, X, X.shape[0], _ptrs(un), _ptrs(uo), alpha, vbar, Xbar, _ptrs(unbar), _ptrs(uobar))

    def advect_vjp(self, u, dt, X, xbar, ubar):
        X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
        u = [np.ascontiguousarray(x, np.float64) for x in u]
        lib().oc_advect_vjp(self.h, _ptrs(u), dt, X, X.shape[0], xbar, _ptrs(ubar))

    def p2g_vjp(self, pos, vel, u, m, ubar, pos_bar, vel_bar):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, np.float64).reshape(-1, 3)
        u = [np.ascontiguousarray(x, np.float64) for x in u]
        m = [np.ascontiguousarray(x, np.float64) for x in m]
        ubar = [np.ascontiguousarray(x, np.float64) for x in ubar]
        lib().oc_p2g_vjp(self.h, pos, vel, pos.shape[0], _ptrs(u), _ptrs(m), _ptrs(ubar), pos_bar, vel_bar)

    def face_sync_vjp(self, ubar):
        ubar = [np.ascontiguousarray(x, np.float64).copy() for x in ubar]
        lib().oc_face_sync_vjp(self.h, *ubar)
        return ubar

    def divergence_vjp(self, bbar, fluid, dt, ubar):
        lib().oc_divergence_vjp(self.h, np.ascontiguousarray(bbar, np.float64), np.ascontiguousarray(fluid, np.uint8),
                                1.0 / dt, *ubar)

    def gradient_vjp(self, dt, ubar, pbar):
        """In place on ubar (wall faces cleared); pbar += gradient^T ubar.  Needs build() of the step."""
        lib().oc_gradient_vjp(self.h, dt, ubar[0], ubar[1], ubar[2], pbar)

    def advect(self, u, dt, X):
        X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
        u = [np.ascontiguousarray(x, np.float64) for x in u]
        out = np.zeros_like(X)
        lib().oc_advect(self.h, _ptrs(u), dt, X, X.shape[0], out)
        return out


def flip_step(O: "Oracle", pos, vel, dt, alpha, gravity, tol=1e-12, max_cycles=200, method="dc", phase=None,
              rho=(1.0, 1.0)):
    """One FLIP step of the FP64 restatement, in the order the GPU step runs: sort -> P2G ->
    T-junction sync -> backup -> gravity -> walls -> divergence -> solve -> gradient -> sync ->
    walls -> G2P -> RK3.  Returns (pos, vel) in sorted order, the sort permutation and details.
    `phase` (per particle, input order) makes it two-phase: beta = 1/rho from the P2G face phase
    with densities rho = (rho0, rho1)."""
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    vel = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
    _, perm = O.particle_keys(pos)
    ps, vs = pos[perm], vel[perm]
    beta = None
    if phase is None:
        u, m, cnt = O.p2g(ps, vs)
    else:
        u, m, cnt, phi = O.p2g_phase(ps, vs, np.asarray(phase, np.float32)[perm])
        beta = O.phase_beta(phi, rho[0], rho[1])
    u = O.face_sync(u)
    uo = [x.copy() for x in u]
    for a in range(3):
        u[a] = u[a] + dt * gravity[a]
    u = O.wall_bc(u)
    fluid = (cnt > 0).astype(np.uint8)
    b = O.divergence(u, fluid, dt)
    O.set_params(mode=0)
    O.build(bbar=beta, fluid=fluid)
    p, hist = O.solve(b, tol=tol, max_cycles=max_cycles, method=method)
    un = O.gradient_update(p, dt, u)
    un = O.wall_bc(O.face_sync(un))
    vnew = O.g2p(ps, un, uo, alpha, vs)
    xnew = O.advect(un, dt, ps.astype(np.float64))
    return xnew, vnew, perm, dict(u_star=u, u_old=uo, u_new=un, p=p, b=b, fluid=fluid, hist=hist, count=cnt,
                                  beta=beta)


# ------------------------------------------------------------------------------------------------
# Differentiable rollout in FP64 (the oracle gradient).  State x, v in particle-id order.
# ------------------------------------------------------------------------------------------------
def flip_step64(O: "Oracle", x, v, dt, alpha, gravity, tol=1e-12, max_cycles=200, fluid=None):
    """One FLIP step on FP64 state, the GPU step's order.  Returns x', v' and the record the VJP
    needs.  `fluid` (optional) replaces the fluid flags derived from the particle counts."""
    u1, m, cnt = O.p2g64(x, v)
    u2 = O.face_sync(u1)
    uo = [a.copy() for a in u2]
    u4 = O.wall_bc([u2[a] + dt * gravity[a] for a in range(3)])
    fl = (cnt > 0).astype(np.uint8) if fluid is None else fluid
    b = O.divergence(u4, fl, dt)
    O.set_params(mode=0)
    O.build(fluid=fl)
    p, _ = O.solve(b, tol=tol, max_cycles=max_cycles)
    u6 = O.wall_bc(O.face_sync(O.gradient_update(p, dt, u4)))
    v2 = O.g2p64(x, u6, uo, alpha, v)
    x2 = O.advect(u6, dt, x)
    return x2, v2, dict(x=x, v=v, u1=u1, m=m, uo=uo, u6=u6, fluid=fl)


def flip_step64_vjp(O: "Oracle", rec, xbar, vbar, dt, alpha, tol=1e-12, max_cycles=200):
    """Adjoint of flip_step64: (xbar', vbar') -> (xbar, vbar)."""
    x, v, u6, uo = rec["x"], rec["v"], rec["u6"], rec["uo"]
    unb, uob = O._faces(), O._faces()
    xb = np.array(xbar, np.float64).reshape(-1, 3)
    O.advect_vjp(u6, dt, x, xb, unb)
    vb = np.array(vbar, np.float64).reshape(-1, 3)
    O.g2p_vjp(x, u6, uo, alpha, vb, xb, unb, uob)
    g = O.face_sync_vjp(O.wall_bc(unb))
    O.set_params(mode=0)
    O.build(fluid=rec["fluid"])
    pbar = np.zeros(int(O.tot0[0]))
    O.gradient_vjp(dt, g, pbar)
    bbar, _ = O.solve(pbar * rec["fluid"], tol=tol, max_cycles=max_cycles)
    O.divergence_vjp(bbar, rec["fluid"], dt, g)
    g = O.wall_bc(g)
    g = O.face_sync_vjp([g[a] + uob[a] for a in range(3)])
    O.p2g_vjp(x, v, rec["u1"], rec["m"], g, xb, vb)
    return xb, vb


def rollout64(O: "Oracle", x0, u0, steps, dt, alpha, gravity, target, tol=1e-12, fluids=None):
    """v0 = MAC sample of u0 at x0, then `steps` FLIP steps; loss = mean |x_N - target|^2."""
    x = np.ascontiguousarray(x0, np.float64).reshape(-1, 3)
    v = O.sample(x, u0)
    recs = []
    for k in range(steps):
        x, v, rec = flip_step64(O, x, v, dt, alpha, gravity, tol, fluid=None if fluids is None else fluids[k])
        recs.append(rec)
    loss = float(((x - target) ** 2).sum(1).mean())
    return loss, x, recs


def rollout64_grad(O: "Oracle", x0, u0, recs, xN, target, dt, alpha, tol=1e-12):
    """d loss / d u0 (three face arrays) by the adjoint of rollout64."""
    n = xN.shape[0]
    xb = 2.0 * (xN - target) / n
    vb = np.zeros_like(xb)
    for rec in reversed(recs):
        xb, vb = flip_step64_vjp(O, rec, xb, vb, dt, alpha, tol)
    ub = O._faces()
    O.sample_vjp(np.ascontiguousarray(x0, np.float64).reshape(-1, 3), u0, vb, ub, None)
    return ub


def grad_along_states(O: "Oracle", xs, vs, u0, target, dt, alpha, gravity, tol=1e-12):
    """d loss / d u0 in FP64 along a given trajectory: xs[k], vs[k] (k = 0..N, particle-id order)
    are the states another implementation produced.  Each step's adjoint is evaluated at that
    step's given input state, so the result isolates the adjoint arithmetic from the divergence of
    two forward trajectories."""
    recs = []
    for k in range(len(xs) - 1):
        _, _, rec = flip_step64(O, np.asarray(xs[k], np.float64), np.asarray(vs[k], np.float64), dt, alpha, gravity, tol)
        rec.pop("u1_sync", None)
        recs.append(rec)
    xN = np.asarray(xs[-1], np.float64)
    n = xN.shape[0]
    xb = 2.0 * (xN - target) / n
    vb = np.zeros_like(xb)
    for rec in reversed(recs):
        xb, vb = flip_step64_vjp(O, rec, xb, vb, dt, alpha, tol)
    ub = O._faces()
    O.sample_vjp(np.asarray(xs[0], np.float64), u0, vb, ub, None)
    return ub
