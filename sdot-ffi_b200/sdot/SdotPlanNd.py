"""`SdotPlanNd`: the solution of a semi-discrete transport in dimension 2 or 3 (src/sdot/SdotPlanNd.py:281-1122).

The whole fit is ONE call of the C ABI (`sdot_solve`, or `sdot_solve_batch` for many problems at once): the
start, the stages, the damped Newton with its diagrams, Laplacians and CG solves, and the final moments all
run on the GPU; Python only sets up the problem and reads what comes out -- the reference's split
(SdotPlanNd.py:1-24).  `stats` and `history` carry the reference's keys in the reference's order.
"""
import numpy as np

from . import _lib
from .PowerDiagram import PowerDiagram

_STATS = ["status", "residual", "residual0", "nb_iter", "nb_diag", "nb_backtracks", "t_majorant", "t_diag", "t_asm", "t_lin", "t_lim", "eps",
          "domain_mass", "nb_overflowed", "nb_cell_lim", "nb_limit_rounds", "lin_nb_hierarchies", "lin_nb_iter", "lin_worst", "start", "t_total",
          "nb_continuation_steps", "min_start_mass", "it_switch", "it_double", "scratch_bytes",
          "nb_clusters", "nb_aggregated", "nb_duplicates", "residual_full", "nb_polish"]
_HISTORY = ["step", "t", "residual_l2", "min_measure", "max_abs_residual", "nb_diag", "nb_evals", "s"]
_STATUS = {0: "running", 1: "converged", 2: "max iterations", 3: "stagnation", 4: "linear solver failure", 5: "card capacity",
           6: "failure", 7: "converged (aggregated)"}
_START = {0: "weights0", 1: "voronoi", 2: "similarity"}
_RESIDUAL = {"lin": 0, "log": 1, "power": 2}
_CONTINUATION = {"never": 0, "auto": 1, "always": 2}
_INT_STATS = ("nb_iter", "nb_diag", "nb_backtracks", "nb_overflowed", "nb_cell_lim", "nb_limit_rounds", "lin_nb_hierarchies", "lin_nb_iter",
              "nb_continuation_steps", "scratch_bytes", "nb_clusters", "nb_aggregated", "nb_duplicates", "nb_polish")


#: the aggregation's margin `kappa` (SdotPlanNd.py:118): a pair is merged when its floor c_ij ulp(w) is within kappa of
#: the tolerance; and the weight gap of an exact duplicate, relative to the cloud's squared extent (SdotPlanNd.py:121)
_AGGREGATE_MARGIN = 4.0

#: `Tuning.step`: the trials of KMT's damping, or the limits of the cells below the floor; "auto" is the limits in 2D and
#: the trials in 3D, as the reference (SdotPlanNd.py:461-462: the engine takes the trials in 3D whatever the option says)
_STEP = {"auto": 1, "trials": 0, "limits": 1}
_DUPLICATE_GAP = 1e-6


def exact_duplicates(positions):
    """`( dup, rep )`: each exact duplicate and the smallest index at its position (SdotPlanNd.py:124-148)"""
    P = np.ascontiguousarray(np.asarray(positions, dtype=np.float64)) + 0.0
    n = P.shape[0]
    none = (np.zeros(0, np.int64), np.zeros(0, np.int64))
    if n < 2:
        return none
    _, idx, inv = np.unique(P.reshape(n, -1), axis=0, return_index=True, return_inverse=True)
    if len(idx) == n:
        return none
    rep = idx[inv.reshape(-1)]
    dup = np.nonzero(rep != np.arange(n))[0]
    return dup.astype(np.int64), rep[dup].astype(np.int64)


def solver_options(settings, n, d=None):
    """the option vector of `sdot_solve_desc` from `Iterative` / `Tuning` (`d`, when given, checks the step against the
    dimension: `limits` is 2D only, SdotPlanNd.py:461-465)"""
    tun = settings.tuning
    if tun.step not in ("auto", "trials", "limits"):
        raise ValueError(f"unknown step : {tun.step!r} ( 'auto', 'trials' or 'limits' )")
    if tun.step == "limits" and d is not None and d != 2:
        raise ValueError("step = 'limits': 2D only (the area polynomials along the direction); in 3D: 'trials' or 'auto'")
    if tun.residual not in _RESIDUAL:
        raise ValueError(f"unknown residual: {tun.residual!r} ( {', '.join(_RESIDUAL)} )")
    if tun.linear_solver not in ("auto", "cg", "mg", "amg"):
        raise NotImplementedError(f"linear_solver = {tun.linear_solver!r}: 'auto' / 'mg' (multigrid-PCG) or 'cg' (Jacobi-PCG) in this build")
    if settings.kernel_dtype == "FP32" and d is not None and d != 2:
        raise NotImplementedError(f"precision = {settings.precision!r}: the FP32 clip is built in 2D; 3D clips in FP64 ( 'fp64' / 'auto' )")
    return dict(tol_abs=settings.tol, tol_rel=float(tun.mass_rtol), maxit=settings.max_iter, max_backtracks=tun.max_backtracks,
                t_min=tun.t_min, mult_ok=tun.restart_factor, residual=_RESIDUAL[tun.residual], power=tun.residual_power,
                switch=tun.residual_switch, lin_tol=float(tun.linear_tol or 1e-6), lin_maxit=int(tun.linear_maxit or 20000),
                keep_start=int(bool(tun.keep_start)), continuation=_CONTINUATION[settings.continuation], conv_threshold=tun.conv_threshold,
                conv_s0=float(tun.conv_start or 0.0), conv_ratio=float(tun.conv_ratio), conv_min=float(tun.conv_min or 0.0),
                lin_method=0 if tun.linear_solver == "cg" else 1, precision=1 if settings.kernel_dtype == "FP32" else 0,
                lin_precision=1 if getattr(tun, "linear_precision", "fp64") == "mixed" else 0,
                agg_margin=(float(_AGGREGATE_MARGIN if tun.aggregation_margin is None else tun.aggregation_margin) if settings.aggregate else 0.0),
                step=0 if tun.step == "auto" and d is not None and d != 2 else _STEP[tun.step])


def _box_of(problem):
    d = problem.nb_dims
    from .PowerDiagram import _domain_box
    return _domain_box(problem.domain, d)


class SdotPlanNd:
    """see the module docstring"""

    @classmethod
    def _solve(cls, problem, settings, verbose=False, warm=None):
        return cls._solve_many([problem], settings, [warm])[0]

    @classmethod
    def _solve_many(cls, problems, settings, warms=None):
        """many problems in ONE batched call (their cells, Laplacians and CG iterations share launches)"""
        warms = warms or [None] * len(problems)
        plans, pbs, opts = [], [], []
        for problem, warm in zip(problems, warms):
            self = cls.__new__(cls)
            self.problem = problem
            src, dst = problem.source, problem.target
            n, d = src.nb_diracs, src.nb_dims
            # EXACT DUPLICATES (sdotplan/Aggregation.h:24-31): each keeps an empty cell (its weight its representative's
            # minus a gap) and its representative (the smallest index at that position) carries its target.  An empty cell
            # cuts no other, so the solve runs on the cloud without them and their outputs are written back after it.
            dup, rep = exact_duplicates(src.positions) if settings.aggregate else (np.zeros(0, np.int64), np.zeros(0, np.int64))
            self._dups = (dup, rep)
            keep = np.setdiff1d(np.arange(n), dup) if len(dup) else None
            self._keep = keep
            plan = settings.ot_plan if settings.ot_plan is not None else warm
            if settings.weights0 is not None:
                w0, self._warm_start = np.asarray(settings.weights0, dtype=np.float64).reshape(-1), "weights0"
            elif plan is not None:
                if len(plan.weights) != n:
                    if settings.ot_plan is not None:
                        raise ValueError(f"Iterative( ot_plan = ... ): this plan carries {len(plan.weights)} weights and the source has {n}")
                    w0, self._warm_start = None, f"none ( the kept plan carries {len(plan.weights)} weights, the source has {n} )"
                else:
                    w0, self._warm_start = plan.weights, "ot_plan"
            else:
                w0, self._warm_start = None, "none"
            lo, hi = _box_of(problem)
            self._box = (lo, hi)
            self._settings = settings
            P, nu = src.positions, src.weights
            if keep is not None:
                nu = np.full(n, 1.0 / n) if nu is None else np.asarray(nu, dtype=np.float64).reshape(-1).copy()
                np.add.at(nu, rep, nu[dup])
                P, nu = P[keep], nu[keep]
                w0 = None if w0 is None else np.asarray(w0, dtype=np.float64).reshape(-1)[keep]
            pbs.append((P, nu, w0, lo, hi, dst._sdot_density()))
            opts.append(solver_options(settings, n, problem.nb_dims))
            plans.append(self)
        results = _lib.solve_batch(pbs, opts, cap_history=8 * (settings.max_iter + 1) + 64)
        for self, r in zip(plans, results):
            if isinstance(r, Exception):
                raise r
            self._read(r, settings)
        for self in plans:
            self._check_converged(settings)
        return plans

    def _expand(self, r):
        """the outputs of the solve without the exact duplicates, written for every seed"""
        dup, rep = self._dups
        keep = self._keep
        P = np.asarray(self.problem.source.positions, dtype=np.float64)
        n, d = P.shape
        w, m, b, cl = np.zeros(n), np.zeros(n), P.copy(), np.arange(n, dtype=np.int64)
        w[keep], m[keep], b[keep] = r["weights"], r["masses"], r["barycentres"]
        cl[keep] = keep[np.asarray(r["clusters"], dtype=np.int64)]
        ext = P.max(axis=0) - P.min(axis=0)
        gap = _DUPLICATE_GAP * max(float((P * P).sum(axis=1).max()), float((ext * ext).sum()), 1e-300)
        count = {}
        for i, j in zip(dup, rep):
            count[j] = count.get(j, 0) + 1
            w[i] = w[j] - gap * count[j]
            cl[i] = cl[j]
        return dict(r, weights=w, masses=m, barycentres=b, clusters=cl)

    def _read(self, r, settings):
        if self._keep is not None:
            r = self._expand(r)
        #: the fitted weights, [n], user order, `weights[ 0 ] == 0`
        self.weights = r["weights"]
        self._weights_fit = self.weights
        #: the mass of each cell at the fitted weights (the one Newton measured)
        self.cell_masses = r["masses"]
        #: the barycentre of each cell [n, d] (its seed if it is empty)
        self.barycenters = r["barycentres"]
        #: the transport cost W2^2
        self.cost = r["cost"]
        st = r["stats"]
        self.stats = {name: float(st[k]) for k, name in enumerate(_STATS)}
        self.stats["status"] = _STATUS.get(int(self.stats["status"]), "?")
        self.stats["it_switch"] = int(self.stats["it_switch"])
        self.stats["it_double"] = int(self.stats["it_double"])
        self.stats["start"] = _START.get(int(self.stats["start"]), "?")
        for name in _INT_STATS:
            self.stats[name] = int(self.stats[name])
        cl = np.asarray(r["clusters"], dtype=np.int64)
        merged = cl != np.arange(len(cl))
        reps = np.unique(cl[merged]) if merged.any() else np.zeros(0, np.int64)
        self._clusters = cl if merged.any() else None
        self.stats["nb_clusters"] = int(len(reps))
        self.stats["nb_aggregated"] = int(merged.sum() + len(reps))
        self.stats["nb_duplicates"] = int(len(self._dups[0]))
        if not settings.aggregate:
            self.stats["aggregation"] = "off"
        else:
            self.stats["aggregation"] = f"{len(reps)} clusters, {self.stats['nb_aggregated']} seeds" if len(reps) else "none"
        self.stats["duplicates"] = "checked" if settings.aggregate else "not checked"
        self.stats["warm_start"] = self._warm_start
        self.history = []
        for row in r["history"]:
            e = {name: float(row[k]) for k, name in enumerate(_HISTORY)}
            e["step"] = int(e["step"])
            self.history.append(e)

    def _check_converged(self, settings):
        if settings.on_failure == "raise" and not self.converged:
            from .OtProblem import OtNotConverged
            raise OtNotConverged(self)

    @property
    def converged(self):
        return self.stats["status"] in ("converged", "converged (aggregated)")

    @property
    def clusters(self):
        """each seed's cluster by its smallest index, or `None` when no seeds were merged (SdotPlanNd.py:629-641)"""
        return self._clusters

    @property
    def target_masses(self):
        nu = self.problem.source.weights
        return nu * (self.stats["domain_mass"] / float(nu.sum()))

    def power_diagram(self, weights=None):
        w = self._weights_fit if weights is None else weights
        return PowerDiagram(self.problem.source.positions, w, boundaries=_box_half(self._box), distribution=self.problem.target)

    def residual(self, weights=None):
        return self.power_diagram(weights).measures - self.target_masses

    def transport(self):
        return self.cost, self.barycenters, self.cell_masses

    def cost_and_position_grad(self):
        """`( cost, grad )`: the derivative of the cost wrt the positions, `2 m_i ( p_i - b_i )` (envelope theorem,
        SdotPlanNd.py:1107-1122)"""
        return self.cost, 2 * self.cell_masses[:, None] * (self.problem.source.positions - self.barycenters)


def _box_half(box):
    from .PowerDiagram import box_half_spaces
    return box_half_spaces(*box)
