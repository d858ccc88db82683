"""`PowerDiagram`: the seeds, their weights and a box domain; cells built on the GPU on demand.

Same constructor and queries as the reference's view (src/sdot/PowerDiagram.py:120-210, 324-496): `measures`,
`moments`, `hessian_rows()`, `laplacian_solve( rhs )`, the `weights` setter.  The cell of seed i is where
`|x - p_i|^2 - w_i` is smallest (PowerDiagram.py:3-10).  Every query is ONE call of the C ABI
(`sdot_cells`, `sdot_laplacian`, `sdot_linear_solve`): the grid index is built on the device, the cells are
clipped one warp per cell, nothing runs on the CPU.  Domains are axis-aligned boxes (`box_half_spaces`);
`cells` / `cell( i )` (display and the reference's slow Python oracle) are not part of this build.
"""
import numpy as np

from . import _lib
from .distributions import Image


def box_half_spaces(mi, ma):
    """the box `mi <= x <= ma` as `2d` half-spaces `direction . x <= offset` (PowerDiagram.py:706-713)"""
    mi = np.asarray(mi, dtype=float).reshape(-1)
    ma = np.asarray(ma, dtype=float).reshape(-1)
    if mi.size != ma.size:
        raise ValueError("`box_half_spaces( mi, ma )` wants two corners of the same dimension")
    d = mi.size
    return np.concatenate([np.eye(d), -np.eye(d)]), np.concatenate([ma, -mi])


def axis_aligned_box(directions, offsets):
    """`( mi, ma, kept )`: the tightest box the axis-aligned half-spaces give and which planes it does NOT
    express (PowerDiagram.py:657-703); `None` if an axis is not bounded on both sides"""
    dirs = np.asarray(directions, dtype=float)
    offs = np.asarray(offsets, dtype=float).reshape(-1)
    if dirs.ndim != 2 or len(dirs) != len(offs):
        return None
    d = dirs.shape[1]
    mi, ma = np.full(d, -np.inf), np.full(d, np.inf)
    for k in range(len(dirs)):
        nz = np.flatnonzero(dirs[k])
        if nz.size != 1:
            continue
        a = int(nz[0])
        c = dirs[k, a]
        if c > 0:
            ma[a] = min(ma[a], offs[k] / c)
        else:
            mi[a] = max(mi[a], offs[k] / c)
    if not np.isfinite(mi).all() or not np.isfinite(ma).all() or not (mi < ma).all():
        return None
    kept = np.ones(len(dirs), dtype=bool)
    for k in range(len(dirs)):
        nz = np.flatnonzero(dirs[k])
        if nz.size != 1:
            continue
        a = int(nz[0])
        c = dirs[k, a]
        kept[k] = offs[k] / c != (ma[a] if c > 0 else mi[a])
    return mi, ma, kept


def _domain_box(boundaries, d):
    if boundaries is None:
        raise NotImplementedError("PowerDiagram: an unbounded domain is not supported here -- give `boundaries` or a distribution with a support")
    box = axis_aligned_box(*boundaries)
    if box is None:
        raise NotImplementedError("PowerDiagram: the domain must be an axis-aligned box (`box_half_spaces`)")
    mi, ma, kept = box
    dirs = np.asarray(boundaries[0], dtype=float).reshape(-1, d)[kept]
    offs = np.asarray(boundaries[1], dtype=float).reshape(-1)[kept]
    # a kept plane that does not cut the box changes nothing; any other is a polytope domain
    corners = np.array(np.meshgrid(*[[mi[a], ma[a]] for a in range(d)], indexing="ij")).reshape(d, -1).T
    for k in range(len(offs)):
        if (corners @ dirs[k] > offs[k] + 1e-14 * (1 + abs(offs[k]))).any():
            raise NotImplementedError("PowerDiagram: the domain must be an axis-aligned box (`box_half_spaces`)")
    return mi, ma


class PowerDiagram:
    def __init__(self, positions, weights=None, boundaries=None, accelerator=None, distribution=None, kernel_dtype=None,
                 scratch_capacity=None, memory=None):
        """`positions` [n, d] (d = 2 or 3), `weights` [n] or None, `boundaries = box_half_spaces( mi, ma )`.
        `distribution`: what to integrate (normalised here, its support intersected with the domain); absent,
        `measures` are volumes.  `accelerator`, `scratch_capacity`, `memory` are accepted for compatibility and
        change nothing (the index is the device-built Morton grid).  `kernel_dtype`: "FP64" (default)."""
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64))
        if pos.ndim != 2:
            raise ValueError(f"`positions` has to be [ n, d ] ( got {tuple(pos.shape)} )")
        n, d = pos.shape
        if d not in (2, 3):
            raise NotImplementedError(f"PowerDiagram: dimension {d} (2 and 3 only here)")
        if distribution is not None:
            distribution = distribution.normalized_version(nb_dims=d)
            if distribution.nb_dims != d:
                raise ValueError(f"the distribution lives in {distribution.nb_dims}D, this diagram in {d}D")
            support = distribution.bounding_half_spaces()
            if support is not None:
                if boundaries is None:
                    boundaries = support
                else:
                    boundaries = (np.concatenate([np.asarray(boundaries[0], float), support[0]]),
                                  np.concatenate([np.asarray(boundaries[1], float), support[1]]))
        self.box_min, self.box_max = _domain_box(boundaries, d)
        self._positions = pos
        self._weights = None if weights is None else np.asarray(weights, dtype=np.float64).reshape(n).copy()
        self.distribution = distribution
        if kernel_dtype not in (None, "FP64", "fp64", "double", "FP32", "fp32", "float"):
            raise ValueError(f"PowerDiagram: unknown kernel_dtype {kernel_dtype!r} ( 'FP64' or 'FP32' )")
        # FP32: the clip in FP32 with FP64 re-checks, the outputs in FP64 (the reference's float kernel); 2D only here
        self._kernel_dtype = "FP32" if kernel_dtype in ("FP32", "fp32", "float") else "FP64"
        if self._kernel_dtype == "FP32" and d != 2:
            raise NotImplementedError("PowerDiagram: kernel_dtype FP32 is built in 2D; 3D clips in FP64")

    # ---- the seeds ----------------------------------------------------------------------------------------
    @property
    def positions(self):
        return self._positions

    @property
    def weights(self):
        return self._weights

    @weights.setter
    def weights(self, w):
        self._weights = None if w is None else np.asarray(w, dtype=np.float64).reshape(self.nb_points).copy()

    @property
    def nb_points(self):
        return self._positions.shape[0]

    @property
    def dim_count(self):
        return self._positions.shape[1]

    def _precision(self):
        return 1 if self._kernel_dtype == "FP32" else 0

    @property
    def kernel_dtype(self):
        return self._kernel_dtype

    def _density(self):
        if self.distribution is None:
            return ("uniform", 1.0)
        return self.distribution._sdot_density()

    # ---- what is read -----------------------------------------------------------------------------------------
    @property
    def measures(self):
        """the measure of each cell, [n], in the order of `positions` (the integral of the distribution if any)"""
        return _lib.cells(self._positions, self._weights, self.box_min, self.box_max, self._density(), precision=self._precision())["masses"]

    @property
    def moments(self):
        """`( masses, first, second )`: int rho, int x rho [n, d], int |x|^2 rho (PowerDiagram.py:448-477)"""
        r = _lib.cells(self._positions, self._weights, self.box_min, self.box_max, self._density(), want_moments=True, precision=self._precision())
        m, b, c = r["masses"], r["barycentres"], r["costs"]
        first = m[:, None] * b
        p = self._positions
        second = c + 2 * (p * first).sum(axis=1) - (p * p).sum(axis=1) * m
        return m, first, second

    def barycenters_and_costs(self):
        """`( masses, barycentres [n, d], costs [n] = int_cell |x - p_i|^2 rho )`, one sweep"""
        r = _lib.cells(self._positions, self._weights, self.box_min, self.box_max, self._density(), want_moments=True, precision=self._precision())
        return r["masses"], r["barycentres"], r["costs"]

    def hessian_rows(self):
        """`( nb_nbrs, ids, vals )`: per cell its seed neighbours and `int_facet rho / ( 2 |p_i - p_j| )`
        (PowerDiagram.py:478-497).  Host arrays."""
        r = _lib.cells(self._positions, self._weights, self.box_min, self.box_max, self._density(), want_facets=True, precision=self._precision())
        return r["nb_count"].astype(int), r["nb_ids"], r["nb_coef"]

    def facets(self):
        """`( nb_nbrs, ids, coef, measure )`: as `hessian_rows`, plus `int_facet rho` (the face length / area for rho = 1)"""
        r = _lib.cells(self._positions, self._weights, self.box_min, self.box_max, self._density(), want_facets=True, precision=self._precision())
        return r["nb_count"].astype(int), r["nb_ids"], r["nb_coef"], r["nb_measure"]

    def laplacian(self):
        """the Laplacian of the Laguerre graph: `( row_ptr, cols, vals, dia )`, CSR in user order, bit-symmetric"""
        return _lib.laplacian(self._positions, self._weights, self.box_min, self.box_max, self._density())

    def laplacian_solve(self, rhs, linear_solver="auto", tol=1e-12):
        """`x = L^+ rhs` with `x[ 0 ] == 0` (PowerDiagram.py:395-430); `rhs` of zero sum.  On the GPU."""
        if linear_solver not in ("auto", "cg"):
            raise NotImplementedError(f"laplacian_solve: linear_solver {linear_solver!r} (auto / cg here)")
        row, cols, vals, dia = self.laplacian()
        x, its = _lib.linear_solve(row, cols, vals, dia, np.asarray(rhs, dtype=np.float64).reshape(1, -1), tol=tol)
        if its[0] < 0:
            raise RuntimeError("laplacian_solve: the CG did not converge")
        return x[0]

    def measures_vjp(self, grad_masses):
        """the adjoint of `measures`: `( grad_positions [n, d], grad_weights [n] )` for the cotangent `grad_masses`"""
        return _lib.cells_vjp(self._positions, self._weights, self.box_min, self.box_max, self._density(), grad_masses)

    def moments_vjp(self, grad_masses=None, grad_first=None):
        """the adjoint of the masses and of the first moments `int_cell x rho` [n, d] (the backward of `moment(k)`, k < d,
        PowerDiagram.py:341-353): `( grad_positions [n, d], grad_weights [n] )`.  A constant density."""
        if grad_first is None:
            return self.measures_vjp(np.zeros(self.nb_points) if grad_masses is None else grad_masses)
        return _lib.cells_vjp(self._positions, self._weights, self.box_min, self.box_max, self._density(), grad_masses, grad_first)


class Voronoi(PowerDiagram):
    """the power diagram without weights"""

    def __init__(self, positions, boundaries=None, **kwargs):
        super().__init__(positions, None, boundaries=boundaries, **kwargs)
