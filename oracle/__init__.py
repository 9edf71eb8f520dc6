"""ORACLE -- test infrastructure only (checker, never the thing measured).

ctypes front-end of ``liboracle.so``, the CPU FP64 restatement of the
reference's transfer path (see ``picasso_oracle.c`` for the file:line of the
reference code each function follows).  Arrays are numpy; particle members
are (N,), (N, C) or (N, R, C) C-contiguous float64 arrays, grid arrays are
(nx, ny, nz[, C]) float64 arrays.  The descriptor structures are the ones of
the public header (shared with the product's ctypes mirror).
"""

import ctypes as C
import os
import subprocess

import numpy as np

from picasso_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        # make is a no-op when the library is up to date with its sources
        build()
        L = C.CDLL(LIB)
        P = C.POINTER
        sig = {
            "oracle_apic_p2g": [P(_abi.Spline), C.c_int64, C.c_int, _abi.ParticleField,
                                _abi.ParticleField, _abi.ParticleField, _abi.GridField,
                                _abi.GridField, P(C.c_int64)],
            "oracle_apic_g2p": [P(_abi.Spline), C.c_int64, C.c_int, _abi.ParticleField,
                                _abi.GridField, _abi.ParticleField, P(C.c_int64)],
            "oracle_polypic_p2g": [P(_abi.Spline), C.c_int64, C.c_int, _abi.ParticleField,
                                   _abi.ParticleField, _abi.ParticleField, _abi.ParticleField,
                                   _abi.GridField, _abi.GridField, C.c_double, P(C.c_int64)],
            "oracle_polypic_g2p": [P(_abi.Spline), C.c_int64, C.c_int, _abi.ParticleField,
                                   _abi.GridField, _abi.ParticleField, P(C.c_int64)],
            "oracle_grid_velocity": [P(_abi.Mesh), C.c_int, _abi.GridField, _abi.GridField,
                                     C.c_double, _abi.GridField],
            "oracle_grid_update": [P(_abi.Mesh), _abi.GridField, _abi.GridField, _abi.GridField,
                                   C.c_double, P(C.c_double), C.c_double, P(C.c_int), C.c_int,
                                   _abi.GridField],
            "oracle_advect": [P(_abi.Mesh), C.c_int64, C.c_double, _abi.ParticleField,
                              _abi.ParticleField],
            "oracle_cell_sort": [P(_abi.Spline), C.c_int64, _abi.ParticleField, P(C.c_int),
                                 C.c_void_p, C.c_void_p, C.c_void_p],
            "oracle_mat3_inverse": [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p],
            "oracle_apic_step_omp": [P(_abi.Spline), C.c_int64, C.c_int, _abi.ParticleField,
                                     _abi.ParticleField, _abi.ParticleField, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_double],
            "oracle_spline": [P(_abi.Spline), C.c_void_p, C.c_void_p],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.oracle_mat3_inverse.restype = None
        _lib = L
    return _lib


def _pf(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    f = _abi.ParticleField()
    f.data = a.ctypes.data
    f.dtype = _abi.F64
    f.vector_shift = 0
    f.tile_stride = int(np.prod(a.shape[1:])) if a.ndim > 1 else 1
    f.comp_stride = 1
    return f


def _gf(a):
    assert a.dtype == np.float64
    g = _abi.GridField()
    g.data = a.ctypes.data
    g.dtype = _abi.F64
    g.fixed_bits = 0
    st = [s // 8 for s in a.strides]
    for d in range(3):
        g.stride[d] = st[d]
    g.stride[3] = st[3] if a.ndim == 4 else 0
    return g


def _check(st, where):
    if st != 0:
        raise RuntimeError("%s: oracle status %d" % (where, st))


def apic_p2g(sd, x, m, c, m_i, mu_i):
    """Adds into m_i / mu_i; returns the number of skipped particles."""
    sk = C.c_int64()
    _check(lib().oracle_apic_p2g(C.byref(sd), x.shape[0], c.shape[2], _pf(x), _pf(m), _pf(c),
                                 _gf(m_i), _gf(mu_i), C.byref(sk)), "apic_p2g")
    return sk.value


def apic_g2p(sd, x, u_i, c):
    sk = C.c_int64()
    _check(lib().oracle_apic_g2p(C.byref(sd), x.shape[0], c.shape[2], _pf(x), _gf(u_i), _pf(c),
                                 C.byref(sk)), "apic_g2p")
    return sk.value


def polypic_p2g(sd, x, m, u, c, mu_i, m_i, dt):
    sk = C.c_int64()
    _check(lib().oracle_polypic_p2g(C.byref(sd), x.shape[0], c.shape[2], _pf(x), _pf(m), _pf(u),
                                    _pf(c), _gf(mu_i), _gf(m_i), float(dt), C.byref(sk)),
           "polypic_p2g")
    return sk.value


def polypic_g2p(sd, x, u_i, c):
    sk = C.c_int64()
    _check(lib().oracle_polypic_g2p(C.byref(sd), x.shape[0], c.shape[2], _pf(x), _gf(u_i), _pf(c),
                                    C.byref(sk)), "polypic_g2p")
    return sk.value


def grid_velocity(mesh, m_i, mu_i, u_i, thr=1e-12):
    nc = mu_i.shape[3] if mu_i.ndim == 4 else 1
    _check(lib().oracle_grid_velocity(C.byref(mesh), nc, _gf(m_i), _gf(mu_i), float(thr),
                                      _gf(u_i)), "grid_velocity")


def grid_update(mesh, m_i, mu_i, u_i, dt, gravity, f_i=None, thr=1e-12, walls=None, width=1):
    """walls: ((lo, hi),) * 3 with 0 none, 1 no-slip, 2 free-slip."""
    w = (C.c_int * 6)(*[(walls[d][s] if walls else 0) for d in range(3) for s in range(2)])
    g = (C.c_double * 3)(*[float(v) for v in gravity])
    fi = _gf(f_i) if f_i is not None else _abi.GridField()
    _check(lib().oracle_grid_update(C.byref(mesh), _gf(m_i), _gf(mu_i), fi, float(dt), g,
                                    float(thr), w, int(width), _gf(u_i)), "grid_update")


def advect(mesh, x, v, dt):
    _check(lib().oracle_advect(C.byref(mesh), x.shape[0], float(dt), _pf(x), _pf(v)), "advect")


def cell_sort(sd, x, tile):
    n = x.shape[0]
    key = np.zeros(max(n, 1), dtype=np.uint32)
    perm = np.zeros(max(n, 1), dtype=np.uint32)
    nt = 1
    m = sd.mesh
    for d in range(3):
        nb = m.own_extent[d] if m.periodic[d] else m.extent[d]
        nt *= -(-nb // tile[d])
    off = np.zeros(nt + 1, dtype=np.int64)
    t3 = (C.c_int * 3)(*tile)
    _check(lib().oracle_cell_sort(C.byref(sd), n, _pf(x), t3, key.ctypes.data, perm.ctypes.data,
                                  off.ctypes.data), "cell_sort")
    return key[:n], perm[:n], off


def mat3_inverse(a, x=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    inv = np.zeros_like(a)
    det = np.zeros(n)
    y = np.zeros((n, 3)) if x is not None else None
    xc = np.ascontiguousarray(x, dtype=np.float64) if x is not None else None
    lib().oracle_mat3_inverse(n, a.ctypes.data, inv.ctypes.data, det.ctypes.data,
                              xc.ctypes.data if x is not None else None,
                              y.ctypes.data if x is not None else None)
    return (inv, det, y) if x is not None else (inv, det)


def apic_step_omp(sd, x, m, c, nthreads, thr=1e-12):
    """P2G -> grid velocity -> G2P on a dense grid of the mesh extent with
    OpenMP (duplicated scatter grids).  c is overwritten; returns
    (grid mass, grid momentum, grid velocity)."""
    ext = tuple(sd.mesh.extent)
    gm = np.zeros(ext)
    gmu = np.zeros(ext + (3,))
    gu = np.zeros(ext + (3,))
    _check(lib().oracle_apic_step_omp(C.byref(sd), x.shape[0], int(nthreads), _pf(x), _pf(m),
                                      _pf(c), gm.ctypes.data, gmu.ctypes.data, gu.ctypes.data,
                                      float(thr)), "apic_step_omp")
    return gm, gmu, gu


class SplineData(C.Structure):
    _fields_ = [("order", C.c_int), ("nk", C.c_int), ("s", (C.c_int * 4) * 3),
                ("w", (C.c_double * 4) * 3), ("g", (C.c_double * 4) * 3),
                ("d", (C.c_double * 4) * 3), ("dx", C.c_double * 3), ("x0", C.c_double * 3)]


def spline(sd, xp):
    out = SplineData()
    xa = (C.c_double * 3)(*xp)
    _check(lib().oracle_spline(C.byref(sd), C.cast(xa, C.c_void_p), C.cast(C.pointer(out), C.c_void_p)),
           "spline")
    k = out.nk
    return {"s": np.array([[out.s[d][n] for n in range(k)] for d in range(3)]),
            "w": np.array([[out.w[d][n] for n in range(k)] for d in range(3)]),
            "g": np.array([[out.g[d][n] for n in range(k)] for d in range(3)]),
            "d": np.array([[out.d[d][n] for n in range(k)] for d in range(3)]),
            "dx": np.array(list(out.dx))}
