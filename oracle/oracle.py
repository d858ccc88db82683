"""ORACLE -- test infrastructure, NOT the product.

ctypes wrapper of `libsdot_oracle.so`, the FP64 CPU restatement of the reference's SDOT path
(`sdot_oracle.c` states what it restates and where from).  Only the tests, `__graft_entry__.smoke()`
and the `cpu_baseline` / `--impl reference` legs of `bench.py` may import this module.

Parity status: pinned on the reference's known-answer tests (tests/golden/, the closed-form gaussian facet and
moments, the reference's solver tests restated in tests/test_oracle.py) and on independent checks; not pinned against
outputs of the reference itself (it cannot be imported or compiled here).

Densities are passed as tuples:
    ("uniform", rho)
    ("image", origin[2], pixel_size[2], values[nx, ny])      values[i, j], i along x (distributions/Image.py:12-20)
    ("gauss", centres[ng, d], sigmas[ng], masses[ng])         masses = the mass of each gaussian
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

#: the option vector of `od_solve`, in order
OPTIONS = ["tol_abs", "tol_rel", "maxit", "max_backtracks", "t_min", "mult_ok", "residual", "power", "switch", "lin_tol",
           "lin_maxit", "keep_start", "continuation", "conv_threshold", "conv_s0", "conv_ratio", "conv_min", "brute", "cap", "agg_margin"]
DEFAULTS = dict(tol_abs=1e-8, tol_rel=0.0, maxit=100, max_backtracks=60, t_min=1e-10, mult_ok=4.0, residual=1, power=0.5,
                switch=2.0, lin_tol=1e-12, lin_maxit=100000, keep_start=0, continuation=1, conv_threshold=1e-2, conv_s0=0.0,
                conv_ratio=2 ** 0.5, conv_min=0.0, brute=0, cap=64, agg_margin=0.0)
STATS = ["status", "residual", "residual0", "nb_iter", "nb_diag", "nb_backtracks", "t_majorant", "t_diag", "t_asm", "t_lin", "t_lim", "eps",
         "domain_mass", "nb_overflowed", "nb_cell_lim", "nb_limit_rounds", "lin_nb_hierarchies", "lin_nb_iter", "lin_worst", "start", "t_total",
         "nb_continuation_steps", "min_start_mass", "it_switch", "it_double", "scratch_bytes",
         "nb_clusters", "nb_aggregated", "nb_duplicates", "residual_full", "nb_polish"]


def build():
    """compile the oracle (gcc + OpenMP) next to its source"""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libsdot_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.od_cells.restype = ctypes.c_int
        L.od_cells.argtypes = [ctypes.c_int, ctypes.c_long, P, P, P, ctypes.c_int, P, P, ctypes.c_int, P, P, P, ctypes.c_int, P, P, P, P, P, P]
        L.od_cells_rows.restype = ctypes.c_int
        L.od_cells_rows.argtypes = [ctypes.c_int, ctypes.c_long, P, P, P, ctypes.c_int, P, P, ctypes.c_long, P, P, P, P, ctypes.c_int, P, P, P,
                                    P, P, P]
        L.od_solve.restype = ctypes.c_int
        L.od_solve.argtypes = [ctypes.c_int, ctypes.c_long, P, P, P, P, ctypes.c_int, P, P, P, P, P, P, P, P, P, ctypes.c_long, P, P]
        L.od_laplacian_solve.restype = ctypes.c_int
        L.od_laplacian_solve.argtypes = [ctypes.c_long, ctypes.c_int, P, P, P, P, P, ctypes.c_double, ctypes.c_int]
        L.od_max_threads.restype = ctypes.c_int
        L.od_set_threads.argtypes = [ctypes.c_int]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def encode_density(density, dim):
    """(kind, params, values) as the C side reads them"""
    if density is None:
        density = ("uniform", 1.0)
    kind = density[0]
    if kind == "uniform":
        return 0, np.array([float(density[1])]), np.zeros(1)
    if kind == "image":
        origin, step, values = density[1], density[2], np.asarray(density[3], dtype=np.float64)
        if dim != 2:
            raise NotImplementedError("oracle: images in 2D only")
        nx, ny = values.shape
        par = np.array([origin[0], origin[1], step[0], step[1], nx, ny], dtype=np.float64)
        return 1, par, np.ascontiguousarray(values.reshape(-1))
    if kind == "gauss":
        c = np.asarray(density[1], dtype=np.float64).reshape(-1, dim)
        s = np.asarray(density[2], dtype=np.float64).reshape(-1, 1)
        m = np.asarray(density[3], dtype=np.float64).reshape(-1, 1)
        return 2, np.array([float(len(c))]), np.ascontiguousarray(np.concatenate([c, s, m], axis=1).reshape(-1))
    raise ValueError(f"unknown density {kind!r}")


def cells(pos, weights=None, box=None, density=None, brute=False, cap=64, want=("mass", "bary", "cost", "facets")):
    """one diagram: dict with `mass`, `bary`, `cost`, `nb`, `nid`, `nc` (c_ij), `nm` (int_facet rho), `nvert`, `status`, `bad`;
    the outputs not in `want` are None (3D gaussians: `want=("facets",)` skips the volume quadrature)"""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n, d = pos.shape
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    if box is None:
        box = (np.zeros(d), np.ones(d))
    bx = np.ascontiguousarray(np.concatenate([np.asarray(box[0], float), np.asarray(box[1], float)]))
    kind, par, val = encode_density(density, d)
    out = {k: None for k in ("mass", "bary", "cost", "nb", "nid", "nc", "nm")}
    if "mass" in want:
        out["mass"] = np.zeros(n)
    if "bary" in want:
        out["bary"] = np.zeros((n, d))
    if "cost" in want:
        out["cost"] = np.zeros(n)
    if "facets" in want:
        out["nb"] = np.zeros(n, dtype=np.int32)
        out["nid"] = np.zeros((n, cap), dtype=np.int32)
        out["nc"] = np.zeros((n, cap))
        out["nm"] = np.zeros((n, cap))
    out["nvert"] = np.zeros(n, dtype=np.int32)
    bad = ctypes.c_long(-1)
    st = lib().od_cells(d, n, _p(pos), _p(w), _p(bx), kind, _p(par), _p(val), int(bool(brute)), _p(out["mass"]), _p(out["bary"]),
                        _p(out["cost"]), cap, _p(out["nb"]), _p(out["nid"]), _p(out["nc"]), _p(out["nm"]), _p(out["nvert"]),
                        ctypes.byref(bad))
    out["status"], out["bad"] = st, bad.value
    return out


def cells_rows(pos, rows, weights=None, box=None, density=None, cap=64):
    """the cells `rows` of the diagram of all of `pos` (the same outputs as `cells`, one row per entry of `rows`)"""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n, d = pos.shape
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    k = len(rows)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    if box is None:
        box = (np.zeros(d), np.ones(d))
    bx = np.ascontiguousarray(np.concatenate([np.asarray(box[0], float), np.asarray(box[1], float)]))
    kind, par, val = encode_density(density, d)
    out = dict(mass=np.zeros(k), bary=np.zeros((k, d)), cost=np.zeros(k), nb=np.zeros(k, dtype=np.int32), nid=np.zeros((k, cap), dtype=np.int32),
               nc=np.zeros((k, cap)), nm=np.zeros((k, cap)), nvert=np.zeros(k, dtype=np.int32))
    bad = ctypes.c_long(-1)
    st = lib().od_cells_rows(d, n, _p(pos), _p(w), _p(bx), kind, _p(par), _p(val), k, _p(rows), _p(out["mass"]), _p(out["bary"]),
                             _p(out["cost"]), cap, _p(out["nb"]), _p(out["nid"]), _p(out["nc"]), _p(out["nm"]), _p(out["nvert"]),
                             ctypes.byref(bad))
    out["status"], out["bad"] = st, bad.value
    return out


def laplacian_solve(nb, nid, nc, b, tol=1e-14, maxit=100000):
    nb = np.ascontiguousarray(nb, dtype=np.int32)
    nid = np.ascontiguousarray(nid, dtype=np.int32)
    nc = np.ascontiguousarray(nc, dtype=np.float64)
    n, cap = nid.shape
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n)
    it = lib().od_laplacian_solve(n, cap, _p(nb), _p(nid), _p(nc), _p(b), _p(x), tol, maxit)
    return x, it


def solve(pos, nu=None, box=None, density=None, w0=None, max_steps=None, **options):
    """the damped Newton: dict with `weights`, `masses`, `bary`, `cost`, `stats` (names), `history` (rows), `status`"""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n, d = pos.shape
    nu = np.full(n, 1.0 / n) if nu is None else np.ascontiguousarray(nu, dtype=np.float64)
    if box is None:
        box = (np.zeros(d), np.ones(d))
    bx = np.ascontiguousarray(np.concatenate([np.asarray(box[0], float), np.asarray(box[1], float)]))
    kind, par, val = encode_density(density, d)
    o = dict(DEFAULTS)
    for k, v in options.items():
        if k not in o:
            raise TypeError(f"unknown oracle option {k!r}")
        o[k] = v
    opts = np.array([float(o[k]) for k in OPTIONS])
    w0a = None if w0 is None else np.ascontiguousarray(w0, dtype=np.float64)
    cap_steps = int(max_steps or (int(o["maxit"]) + 1) * 8)
    hist = np.zeros((cap_steps, 8))
    nb_steps = ctypes.c_long(0)
    clusters = np.zeros(n, dtype=np.int32)
    weights, masses, bary, cost, stats = np.zeros(n), np.zeros(n), np.zeros((n, d)), np.zeros(1), np.zeros(len(STATS))
    st = lib().od_solve(d, n, _p(pos), _p(nu), _p(w0a), _p(bx), kind, _p(par), _p(val), _p(opts), _p(weights), _p(masses), _p(bary),
                        _p(cost), _p(stats), _p(hist), cap_steps, ctypes.byref(nb_steps), _p(clusters))
    return dict(weights=weights, masses=masses, bary=bary, cost=float(cost[0]), stats=dict(zip(STATS, stats.tolist())),
                history=hist[:nb_steps.value].copy(), status=st, clusters=clusters)


def max_threads():
    return lib().od_max_threads()


def set_threads(t):
    lib().od_set_threads(int(t))
