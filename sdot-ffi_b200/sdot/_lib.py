"""ctypes binding of `libsdot_b200.so` (the C ABI declared in include/sdot_b200.h).

This plays the part of the reference's FFI layer (`loom.ffi_call`, docs/guide/ffi-internals.md:1-126): it
owns the device contexts, marshals host arrays, and turns the library's `sdot_status` into the exceptions the
reference raises (`KernelFailure` for a cell past its capacity, PowerDiagram_Bsp.py:133-138; `MemoryError`
for a refused pool, CardMemory.py:161-190).  There is no CPU fallback: without the library or a CUDA device
every call raises.
"""
import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libsdot_b200.so")

SDOT_OK, SDOT_ERR_ARGS, SDOT_ERR_CUDA, SDOT_ERR_NO_MEMORY, SDOT_ERR_CAPACITY, SDOT_ERR_UNSUPPORTED, SDOT_ERR_NOT_CONVERGED, SDOT_ERR_TOPOLOGY = range(8)
SDOT_HOST, SDOT_DEVICE = 0, 1
DENSITY_UNIFORM, DENSITY_IMAGE, DENSITY_GAUSSIANS = 0, 1, 2

OPTIONS = ["tol_abs", "tol_rel", "maxit", "max_backtracks", "t_min", "mult_ok", "residual", "power", "switch", "lin_tol", "lin_maxit",
           "keep_start", "continuation", "conv_threshold", "conv_s0", "conv_ratio", "conv_min", "lin_method", "precision", "lin_precision",
           "agg_margin", "step"]
NB_OPTIONS = len(OPTIONS)
NB_STATS = 31
NB_HIST = 8


class KernelFailure(RuntimeError):
    """a cell the kernel could not build (past its vertex / neighbour capacity); `seed` is its user index"""

    def __init__(self, message, seed=-1, needed=0):
        super().__init__(message)
        self.seed = seed
        self.needed = needed


class Status(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int32), ("kind", ctypes.c_int32), ("id", ctypes.c_int64), ("value", ctypes.c_int64),
                ("needed", ctypes.c_int64), ("message", ctypes.c_char * 160)]


class Density(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("value", ctypes.c_double), ("shape", ctypes.c_int32 * 3), ("origin", ctypes.c_double * 3),
                ("step", ctypes.c_double * 3), ("values", ctypes.c_void_p), ("count", ctypes.c_int32), ("centres", ctypes.c_void_p),
                ("sigmas", ctypes.c_void_p), ("masses", ctypes.c_void_p)]


class DiagramDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int32), ("n", ctypes.c_int64), ("positions", ctypes.c_void_p), ("weights", ctypes.c_void_p),
                ("box_lo", ctypes.c_double * 3), ("box_hi", ctypes.c_double * 3), ("density", Density), ("memory", ctypes.c_int32)]


class CellsOut(ctypes.Structure):
    _fields_ = [("masses", ctypes.c_void_p), ("barycentres", ctypes.c_void_p), ("costs", ctypes.c_void_p), ("cap", ctypes.c_int32),
                ("nb_count", ctypes.c_void_p), ("nb_ids", ctypes.c_void_p), ("nb_coef", ctypes.c_void_p), ("nb_measure", ctypes.c_void_p),
                ("precision", ctypes.c_int32)]


class SolveDesc(ctypes.Structure):
    _fields_ = [("diagram", DiagramDesc), ("nu", ctypes.c_void_p), ("options", ctypes.c_double * NB_OPTIONS)]


class SolveOut(ctypes.Structure):
    _fields_ = [("weights", ctypes.c_void_p), ("masses", ctypes.c_void_p), ("barycentres", ctypes.c_void_p), ("cost", ctypes.c_void_p),
                ("stats", ctypes.c_double * NB_STATS), ("history", ctypes.c_void_p), ("cap_history", ctypes.c_int32),
                ("nb_history", ctypes.c_int32), ("clusters", ctypes.c_void_p)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("memory_budget", ctypes.c_uint64), ("max_active", ctypes.c_int32)]


#: every symbol include/sdot_b200.h declares, with its signature
_P = ctypes.c_void_p
SIGNATURES = {
    "sdot_abi_version": (ctypes.c_int32, []),
    "sdot_context_create": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(_P), ctypes.POINTER(Status)]),
    "sdot_context_destroy": (None, [_P]),
    "sdot_context_stream": (_P, [_P]),
    "sdot_context_synchronize": (ctypes.c_int32, [_P, ctypes.POINTER(Status)]),
    "sdot_context_kernel_launches": (ctypes.c_uint64, [_P]),
    "sdot_context_set_timing": (ctypes.c_int32, [_P, ctypes.c_int32]),
    "sdot_context_set_counters": (ctypes.c_int32, [_P, ctypes.c_int32]),
    "sdot_context_gather_counters": (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32]),
    "sdot_context_memory": (ctypes.c_int32, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                             ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32]),
    "sdot_context_kernel_stats": (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64),
                                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int32]),
    "sdot_cells": (ctypes.c_int32, [_P, ctypes.POINTER(DiagramDesc), ctypes.POINTER(CellsOut), ctypes.POINTER(Status)]),
    "sdot_cells_vjp": (ctypes.c_int32, [_P, ctypes.POINTER(DiagramDesc), _P, _P, _P, ctypes.POINTER(Status)]),
    "sdot_cells_vjp_moments": (ctypes.c_int32, [_P, ctypes.POINTER(DiagramDesc), _P, _P, _P, _P, ctypes.POINTER(Status)]),
    "sdot_laplacian": (ctypes.c_int32, [_P, ctypes.POINTER(DiagramDesc), ctypes.c_int64, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(Status)]),
    "sdot_linear_solve": (ctypes.c_int32, [_P, ctypes.c_int64, _P, _P, _P, _P, ctypes.c_int32, _P, _P, ctypes.c_int32, ctypes.c_double,
                                           ctypes.c_int32, ctypes.c_int32, _P, ctypes.POINTER(Status)]),
    "sdot_linear_solve_noalloc": (ctypes.c_int32, [_P, ctypes.c_int64, _P, _P, _P, _P, ctypes.c_int32, _P, _P, ctypes.c_double,
                                                   ctypes.c_int32, _P, ctypes.POINTER(Status)]),
    "sdot_solve": (ctypes.c_int32, [_P, ctypes.POINTER(SolveDesc), ctypes.POINTER(SolveOut), ctypes.POINTER(Status)]),
    "sdot_solve_batch": (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.POINTER(SolveDesc), ctypes.POINTER(SolveOut), ctypes.POINTER(Status)]),
    "sdot_solve_bytes": (ctypes.c_uint64, [ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(Density)]),
    "sdot_w2_backward": (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, _P, ctypes.c_int32, _P, _P, _P, _P, _P, _P,
                                          ctypes.POINTER(Status)]),
    "sdot_server_create": (ctypes.c_int32, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_P), ctypes.POINTER(Status)]),
    "sdot_server_submit": (ctypes.c_int32, [_P, ctypes.POINTER(SolveDesc), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(Status)]),
    "sdot_server_poll": (ctypes.c_int32, [_P, ctypes.c_int64, ctypes.POINTER(SolveOut), ctypes.c_int32, ctypes.POINTER(Status)]),
    "sdot_server_counters": (ctypes.c_int32, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "sdot_server_destroy": (None, [_P]),
}

_lib = None
_lock = threading.Lock()
_contexts = {}


def load():
    """the library, loaded once; raises if it was not built (no fallback)"""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(f"libsdot_b200.so is not built ({LIB_PATH}): run `python sdot-ffi_b200/build.py`")
                L = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def raise_for(code, st, what="sdot"):
    if code == SDOT_OK:
        return
    msg = f"{what}: {st.message.decode(errors='replace')}"
    if code == SDOT_ERR_CAPACITY:
        raise KernelFailure(msg + f" -- seed {st.id} needs {st.needed}", seed=int(st.id), needed=int(st.needed))
    if code == SDOT_ERR_TOPOLOGY:
        raise KernelFailure(msg + f" -- seed {st.id}", seed=int(st.id), needed=0)
    if code == SDOT_ERR_NO_MEMORY:
        raise MemoryError(msg)
    if code == SDOT_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if code == SDOT_ERR_ARGS:
        raise ValueError(msg)
    raise RuntimeError(msg)


def device_index():
    return int(os.environ.get("SDOT_DEVICE", "0"))


def context(device=None):
    """the process's context on `device` (created on first use)"""
    dev = device_index() if device is None else int(device)
    ctx = _contexts.get(dev)
    if ctx is None:
        with _lock:
            ctx = _contexts.get(dev)
            if ctx is None:
                L = load()
                h = ctypes.c_void_p()
                st = Status()
                raise_for(L.sdot_context_create(dev, 0, ctypes.byref(h), ctypes.byref(st)), st, "sdot_context_create")
                ctx = _contexts[dev] = h
    return ctx


def new_context(device=None, pool_limit=0):
    """a context of its own (not the process's), its pool limited to `pool_limit` bytes (0: no limit); free it with
    `destroy_context`"""
    L = load()
    h = ctypes.c_void_p()
    st = Status()
    dev = device_index() if device is None else int(device)
    raise_for(L.sdot_context_create(dev, int(pool_limit), ctypes.byref(h), ctypes.byref(st)), st, "sdot_context_create")
    return h


def destroy_context(h):
    load().sdot_context_destroy(h)


def context_memory(ctx=None, reset_peak=False):
    """the context's pool: bytes in use, the peak since the last reset, and the limit (0: none)"""
    u, p, l = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    code = load().sdot_context_memory(ctx or context(), ctypes.byref(u), ctypes.byref(p), ctypes.byref(l), int(bool(reset_peak)))
    raise_for(code, Status(), "sdot_context_memory")
    return dict(in_use=int(u.value), peak=int(p.value), limit=int(l.value))


def solve_bytes(dim, n, dens):
    """the memory model of one solve (sdot_solve_bytes, the reference's CardMemory.card_solve_bytes)"""
    keep = []
    D = density_struct(dens, keep)
    return int(load().sdot_solve_bytes(int(dim), int(n), ctypes.byref(D)))


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def density_struct(dens, keep):
    """`dens` = (kind, params) from a distribution's `_sdot_density`; arrays are kept alive in `keep`"""
    D = Density()
    kind = dens[0]
    if kind == "uniform":
        D.kind, D.value = DENSITY_UNIFORM, float(dens[1])
    elif kind == "image":
        _, origin, step, values = dens
        v = f64(values)
        keep.append(v)
        D.kind = DENSITY_IMAGE
        D.shape[0], D.shape[1] = v.shape[0], v.shape[1]
        for a in range(2):
            D.origin[a], D.step[a] = float(origin[a]), float(step[a])
        D.values = v.ctypes.data
    elif kind == "gauss":
        _, c, s, m = dens
        c, s, m = f64(c), f64(s).reshape(-1), f64(m).reshape(-1)
        keep.extend([c, s, m])
        D.kind, D.count = DENSITY_GAUSSIANS, len(s)
        D.centres, D.sigmas, D.masses = c.ctypes.data, s.ctypes.data, m.ctypes.data
    else:
        raise ValueError(f"unknown density {kind!r}")
    return D


def diagram_desc(pos, weights, lo, hi, dens, keep, memory=SDOT_HOST):
    desc = DiagramDesc()
    n, d = pos.shape
    desc.dim, desc.n = d, n
    desc.positions = pos.ctypes.data
    desc.weights = None if weights is None else weights.ctypes.data
    for a in range(d):
        desc.box_lo[a], desc.box_hi[a] = float(lo[a]), float(hi[a])
    desc.density = density_struct(dens, keep)
    desc.memory = memory
    keep.extend([pos, weights])
    return desc


def cells(pos, weights, lo, hi, dens, want_facets=False, want_moments=False, cap=None, precision=0):
    """one diagram on the GPU; host arrays in and out.  A cell with more facets than the table's row is reported
    with the capacity it needs, and the call runs again with that capacity (PowerDiagram.py:198-215).  `precision` 1:
    the clip in FP32 with FP64 re-checks (2D)"""
    while True:
        try:
            return _cells_once(pos, weights, lo, hi, dens, want_facets, want_moments, cap, precision)
        except KernelFailure as e:
            grown = max(int(e.needed), 2 * (cap or 32))
            if not want_facets or e.needed <= (cap or 0) or grown > 8192:
                raise
            cap = grown


def _cells_once(pos, weights, lo, hi, dens, want_facets=False, want_moments=False, cap=None, precision=0):
    L = load()
    keep = []
    pos = f64(pos)
    n, d = pos.shape
    w = None if weights is None else f64(weights).reshape(-1)
    desc = diagram_desc(pos, w, lo, hi, dens, keep)
    out = CellsOut()
    out.precision = int(precision)
    res = {"masses": np.zeros(n)}
    out.masses = res["masses"].ctypes.data
    if want_moments:
        res["barycentres"], res["costs"] = np.zeros((n, d)), np.zeros(n)
        out.barycentres, out.costs = res["barycentres"].ctypes.data, res["costs"].ctypes.data
    if want_facets:
        cap = cap or (32 if d == 2 else 64)
        res["nb_count"] = np.zeros(n, np.int32)
        res["nb_ids"] = np.full((n, cap), -1, np.int32)
        res["nb_coef"] = np.zeros((n, cap))
        res["nb_measure"] = np.zeros((n, cap))
        out.cap = cap
        out.nb_count, out.nb_ids = res["nb_count"].ctypes.data, res["nb_ids"].ctypes.data
        out.nb_coef, out.nb_measure = res["nb_coef"].ctypes.data, res["nb_measure"].ctypes.data
    st = Status()
    raise_for(L.sdot_cells(context(), ctypes.byref(desc), ctypes.byref(out), ctypes.byref(st)), st, "sdot_cells")
    return res


def cells_vjp(pos, weights, lo, hi, dens, grad_masses, grad_first=None):
    """(grad_positions [n, d], grad_weights [n]) for the cotangents of the masses [n] and / or (sdot_cells_vjp_moments)
    of the first moments int_cell x rho [n, d]"""
    L = load()
    keep = []
    pos = f64(pos)
    n, d = pos.shape
    w = None if weights is None else f64(weights).reshape(-1)
    desc = diagram_desc(pos, w, lo, hi, dens, keep)
    g = None if grad_masses is None else f64(grad_masses).reshape(-1)
    gp, gw = np.zeros((n, d)), np.zeros(n)
    st = Status()
    if grad_first is None:
        raise_for(L.sdot_cells_vjp(context(), ctypes.byref(desc), ptr(g), ptr(gp), ptr(gw), ctypes.byref(st)), st, "sdot_cells_vjp")
    else:
        gf = f64(grad_first).reshape(n, d)
        raise_for(L.sdot_cells_vjp_moments(context(), ctypes.byref(desc), None if g is None else ptr(g), ptr(gf), ptr(gp), ptr(gw),
                                           ctypes.byref(st)), st, "sdot_cells_vjp_moments")
    return gp, gw


def laplacian(pos, weights, lo, hi, dens):
    """CSR of the Laplacian (user order): row_ptr int64, cols int32, vals (c_ij > 0), dia"""
    L = load()
    keep = []
    pos = f64(pos)
    n, d = pos.shape
    w = None if weights is None else f64(weights).reshape(-1)
    desc = diagram_desc(pos, w, lo, hi, dens, keep)
    cap = n * (32 if d == 2 else 64)
    row = np.zeros(n + 1, np.int64)
    cols = np.zeros(cap, np.int32)
    vals = np.zeros(cap)
    dia = np.zeros(n)
    nnz = ctypes.c_int64(0)
    st = Status()
    raise_for(L.sdot_laplacian(context(), ctypes.byref(desc), cap, ptr(row), ptr(cols), ptr(vals), ptr(dia), ctypes.byref(nnz), ctypes.byref(st)),
              st, "sdot_laplacian")
    k = nnz.value
    return row, cols[:k].copy(), vals[:k].copy(), dia


def linear_solve(row, cols, vals, dia, rhs, tol=1e-10, maxit=100000, method=0):
    L = load()
    row = np.ascontiguousarray(row, np.int64)
    cols = np.ascontiguousarray(cols, np.int32)
    vals, dia = f64(vals), f64(dia)
    rhs = np.atleast_2d(f64(rhs))
    k, n = rhs.shape
    x = np.zeros((k, n))
    its = np.zeros(k, np.int32)
    st = Status()
    raise_for(L.sdot_linear_solve(context(), n, ptr(row), ptr(cols), ptr(vals), ptr(dia), k, ptr(rhs), ptr(x), int(method), float(tol),
                                  int(maxit), SDOT_HOST, ptr(its), ctypes.byref(st)), st, "sdot_linear_solve")
    return x, its


def solve_desc(pos, nu, w0, lo, hi, dens, options, keep):
    pos = f64(pos)
    sd = SolveDesc()
    w = None if w0 is None else f64(w0).reshape(-1)
    sd.diagram = diagram_desc(pos, w, lo, hi, dens, keep)
    nu = None if nu is None else f64(nu).reshape(-1)
    keep.append(nu)
    sd.nu = None if nu is None else nu.ctypes.data
    for k, name in enumerate(OPTIONS):
        sd.options[k] = float(options[name])
    return sd


def solve_out(n, d, cap_history, keep):
    so = SolveOut()
    res = dict(weights=np.zeros(n), masses=np.zeros(n), barycentres=np.zeros((n, d)), cost=np.zeros(1),
               history=np.zeros((max(cap_history, 1), NB_HIST)), clusters=np.zeros(n, np.int32))
    keep.append(res)
    so.weights, so.masses = res["weights"].ctypes.data, res["masses"].ctypes.data
    so.clusters = res["clusters"].ctypes.data
    so.barycentres, so.cost = res["barycentres"].ctypes.data, res["cost"].ctypes.data
    so.history, so.cap_history = res["history"].ctypes.data, cap_history
    return so, res


def solve_batch(problems, options_list, cap_history=512, ctx=None):
    """`problems`: list of (pos, nu, w0, lo, hi, dens); returns a list of result dicts (or exceptions); `ctx`: a context of
    `new_context` (default: the process's)"""
    L = load()
    keep = []
    count = len(problems)
    descs = (SolveDesc * count)()
    outs = (SolveOut * count)()
    results = []
    for k, (pb, opts) in enumerate(zip(problems, options_list)):
        pos = f64(pb[0])
        descs[k] = solve_desc(pos, pb[1], pb[2], pb[3], pb[4], pb[5], opts, keep)
        so, res = solve_out(pos.shape[0], pos.shape[1], cap_history, keep)
        outs[k] = so
        results.append(res)
    sts = (Status * count)()
    L.sdot_solve_batch(ctx or context(), count, descs, outs, sts)
    final = []
    for k in range(count):
        if sts[k].code != SDOT_OK:
            try:
                raise_for(sts[k].code, sts[k], "sdot_solve")
            except Exception as e:          # noqa: BLE001 - handed to the caller per problem
                final.append(e)
                continue
        r = results[k]
        r["stats"] = np.array(outs[k].stats[:])
        r["history"] = r["history"][:outs[k].nb_history].copy()
        r["cost"] = float(r["cost"][0])
        final.append(r)
    return final


def kernel_launches():
    return int(load().sdot_context_kernel_launches(context()))


KERNEL_CLASSES = ["cells2d", "cells3d", "laplacian", "cg", "vector", "index", "report", "multigrid"]


def set_timing(on=True):
    load().sdot_context_set_timing(context(), int(bool(on)))


def kernel_stats(reset=False):
    """{class: (ms, launches, units)} accumulated since the last reset (CUDA events on the context's stream)"""
    L = load()
    res = {}
    for k, name in enumerate(KERNEL_CLASSES):
        ms, n, u = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_double()
        L.sdot_context_kernel_stats(context(), k, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(u), 0)
        res[name] = (ms.value, n.value, u.value)
    if reset:
        L.sdot_context_kernel_stats(context(), 0, None, None, None, 1)
    return res


GATHER_KINDS = ("cells", "candidates", "grid_cells", "grid_ranges", "nodes")


def set_counters(on=True):
    """count the neighbour search's record reads of every `cells` call (sdot_context_set_counters)"""
    load().sdot_context_set_counters(context(), int(bool(on)))


def gather_counters(dim, reset=False):
    """{kind: count} of the `dim`-D diagrams since the last reset (sdot_context_gather_counters)"""
    c = (ctypes.c_uint64 * 5)()
    code = load().sdot_context_gather_counters(context(), int(dim), c, int(bool(reset)))
    if code:
        raise RuntimeError(f"sdot_context_gather_counters: code {code}")
    return dict(zip(GATHER_KINDS, (int(x) for x in c)))


def stream():
    return load().sdot_context_stream(context())
