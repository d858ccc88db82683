"""`OtProblem` / `Iterative` / `Tuning` / `ot_solve`: the reference's entry points of the transport
(src/sdot/OtProblem.py:62-452), same names, keywords and defaults.  A problem holds the two distributions;
`solve` returns an `SdotPlanNd` and keeps it as the warm start of the next solve of the same problem.

Differences of this build, each refused loudly rather than ignored: 1D (`Direct`) is not here; `step = "limits"`,
the aggregation of near-coincident seeds and `precision = "fp32" / "mixed"` are not built yet (the FP64 cells of a
B200 run at half its FP32 rate, so `"auto"` is FP64 on the device as well).
"""
import copy

import numpy as np

_PRECISIONS = {"auto": "FP64", "fp64": "FP64", "fp32": "FP32", "mixed": "FP32"}


class Tuning:
    """the bench settings (OtProblem.py:62-130), same names and defaults; those this build has no use for are
    accepted and ignored only where they cannot change the result (accelerator, memory, scratch_capacity)"""

    def __init__(self, step="auto", linear_solver="auto", amg_variant="auto", linear_tol=None,
                 mg_pack=None, mg_recycle=None, mg_rebuild=None, mg_stop=None, mg_nu=None,
                 mg_kcycle=None, linear_host=False, mg_precision=None, mg_smoothed=None,
                 conv_start=None, conv_ratio=2 ** 0.5, conv_min=None, conv_threshold=1e-2,
                 t_min=1e-10, max_backtracks=60, restart_factor=4.0, mass_rtol=0.0,
                 residual="log", residual_power=0.5, residual_switch=2.0,
                 aggregation_margin=None, accelerator=None, memory=None, scratch_capacity=None, keep_start=False,
                 linear_maxit=None, linear_precision="fp64"):
        self.step = step
        self.linear_solver = linear_solver
        self.amg_variant = amg_variant
        self.linear_tol = linear_tol
        self.mg_pack, self.mg_recycle, self.mg_rebuild, self.mg_stop, self.mg_nu = mg_pack, mg_recycle, mg_rebuild, mg_stop, mg_nu
        self.mg_kcycle, self.linear_host, self.mg_precision, self.mg_smoothed = mg_kcycle, bool(linear_host), mg_precision, mg_smoothed
        self.conv_start, self.conv_ratio, self.conv_min, self.conv_threshold = conv_start, conv_ratio, conv_min, conv_threshold
        self.t_min, self.max_backtracks, self.restart_factor, self.mass_rtol = t_min, max_backtracks, restart_factor, mass_rtol
        self.residual, self.residual_power, self.residual_switch = residual, residual_power, residual_switch
        self.aggregation_margin = aggregation_margin
        self.keep_start = bool(keep_start)
        self.accelerator, self.memory, self.scratch_capacity = accelerator, memory, scratch_capacity
        self.linear_maxit = linear_maxit
        # this build's: "mixed" runs each Newton system's CG in FP32 (FP32 copies of the Laplacian and of the CG's vectors)
        # inside an FP64 iterative refinement that keeps the solution and the residual in FP64
        if linear_precision not in ("fp64", "mixed"):
            raise ValueError(f"unknown linear_precision : {linear_precision!r} ( 'fp64' or 'mixed' )")
        self.linear_precision = linear_precision


class OtNotConverged(RuntimeError):
    """the solve ended without meeting its tolerance; `solution` is the plan it got to (OtProblem.py:133-146)"""

    def __init__(self, solution):
        st = solution.stats
        hint = ""
        if st["min_start_mass"] <= 0:
            hint = " -- the start already had an EMPTY cell ( the target has no mass where a seed starts )"
        super().__init__(f"the transport did not converge: status '{st['status']}', residual {st['residual']:.3e} after "
                         f"{st['nb_iter']} iterations, start '{st['start']}'{hint}")
        self.solution = solution


class Iterative:
    """the settings of the iterative regime (OtProblem.py:149-238): `tol` is ABSOLUTE in normalised masses"""
    regime = "iterative"

    def __init__(self, tol=1e-8, max_iter=100, ot_plan=None, weights0=None, continuation="auto", precision="auto", aggregate=True,
                 keep_weights=False, tuning=None, on_failure="raise", differentiable="auto"):
        if on_failure not in ("raise", "ignore"):
            raise ValueError(f"unknown on_failure : {on_failure!r} ( 'raise' or 'ignore' )")
        if differentiable not in ("auto", True, False):
            raise ValueError(f"unknown differentiable : {differentiable!r} ( 'auto', True or False )")
        if precision not in _PRECISIONS:
            raise ValueError(f"unknown precision : {precision!r} ( {', '.join(_PRECISIONS)} )")
        if continuation not in ("auto", "always", "never"):
            raise ValueError(f"unknown continuation : {continuation!r} ( 'auto', 'always' or 'never' )")
        if ot_plan is not None and weights0 is not None:
            raise ValueError("Iterative : `ot_plan` AND `weights0` -- there is only one starting point")
        self.on_failure = on_failure
        self.differentiable = differentiable
        self.ot_plan = ot_plan
        self.tol = float(tol)
        self.max_iter = int(max_iter)
        self.weights0 = weights0
        self.continuation = continuation
        self.precision = precision
        self.aggregate = bool(aggregate)
        self.keep_weights = bool(keep_weights)
        self.tuning = tuning or Tuning()

    @property
    def kernel_dtype(self):
        return _PRECISIONS[self.precision]


class OtProblem:
    """the inputs of a transport: a discrete `source` (SumOfDiracs) and a continuous `target`"""

    def __init__(self, source, target):
        if target is None:
            raise ValueError("OtProblem : a target is needed -- it is what gives the domain")
        self._last = None
        self._source = None
        self._target = None
        self.source = source
        self.target = target

    @property
    def source(self):
        return self._source

    @source.setter
    def source(self, source):
        if source is None:
            raise ValueError("OtProblem : a source is needed")
        if not getattr(source, "_is_dirac_source", False):
            raise TypeError(f"OtProblem : {type(source).__name__} is not a discrete source")
        source = source.normalized_version()
        if self._source is not None and source.nb_diracs != self._source.nb_diracs:
            self._last = None
        self._source = source

    @property
    def target(self):
        return self._target

    @target.setter
    def target(self, target):
        if target is None:
            raise ValueError("OtProblem : a target is needed -- it is what gives the domain")
        d = None if self._source is None else self._source.nb_dims
        self._target = target.normalized_version(nb_dims=d)

    @property
    def nb_dims(self):
        return self._source.nb_dims

    @property
    def nb_diracs(self):
        return self._source.nb_diracs

    @property
    def regime(self):
        return "direct" if self.nb_dims == 1 else "iterative"

    @property
    def domain(self):
        support = self._target.bounding_half_spaces()
        if support is None:
            raise ValueError("OtProblem : the support of the target does not bound the domain")
        return support

    def solve(self, settings=None, verbose=False):
        regime = self.regime
        if regime == "direct":
            raise NotImplementedError("OtProblem: the 1D direct regime is not part of this build")
        if settings is None:
            settings = Iterative()
        elif getattr(settings, "regime", None) != regime:
            raise TypeError(f"OtProblem.solve : this problem is solved in regime {regime!r} ( nb_dims = {self.nb_dims} ), so its settings "
                            f"are a `Iterative` and not a `{type(settings).__name__}`")
        from .SdotPlanNd import SdotPlanNd
        sol = SdotPlanNd._solve(self, settings, verbose, warm=self._last)
        self._last = sol
        return sol


def ot_solve(source, target, *, verbose=False, **settings):
    """pose and solve in one expression (OtProblem.py:412-452)"""
    pb = OtProblem(source, target)
    try:
        s = Iterative(**settings)
    except TypeError as e:
        import inspect
        names = [n for n in inspect.signature(Iterative).parameters if n != "self"]
        raise TypeError(f"ot_solve : the settings are those of `Iterative` ( {', '.join(names)} ) -- {e}") from None
    return pb.solve(s, verbose)
