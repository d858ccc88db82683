"""The distributions of the hot path, with the reference's names and normalisation rules
(src/sdot/distributions/SumOfDiracs.py:16-71, Image.py:12-94 and 213-245, SumOfGaussians.py:6-131, Box.py:1-60).

Each one knows its support (`bounding_half_spaces`, the domain of a transport) and how it is handed to the
C ABI (`_sdot_density`).  Only axis-aligned images (a diagonal `frame`, uniform knots) are integrated here.
"""
import numpy as np


class Distribution:
    nb_dims = None

    def normalized_version(self, nb_dims=None):
        return self

    def bounding_half_spaces(self):
        return None


class SumOfDiracs(Distribution):
    """Sum of weighted Dirac masses; `weights` (the target masses of the cells) are normalised to `target_mass`"""
    _is_dirac_source = True

    def __init__(self, positions, weights=None, target_mass=1.0):
        self.positions = np.ascontiguousarray(np.asarray(positions, dtype=np.float64))
        if self.positions.ndim != 2:
            raise ValueError(f"SumOfDiracs: positions has to be [ n, d ] (got {self.positions.shape})")
        self.weights = None if weights is None else np.asarray(weights, dtype=np.float64).reshape(-1)
        self.target_mass = target_mass
        self.nb_dims = self.positions.shape[1]

    @property
    def nb_diracs(self):
        return self.positions.shape[0]

    @property
    def mass(self):
        return float(self.weights.sum()) if self.weights is not None else float(self.target_mass)

    def normalized_version(self, nb_dims=None):
        n = self.nb_diracs
        if self.weights is None:
            w = np.full(n, self.target_mass / n)
        else:
            w = self.target_mass / self.weights.sum() * self.weights
        return SumOfDiracs(self.positions, w, target_mass=self.target_mass)


class Image(Distribution):
    """Piecewise constant on a grid: `values[ i, j ]`, i along x (2D).  `origin` is the corner of pixel (0, 0),
    `frame` the pixel edges (a diagonal matrix or a vector of sizes; identity by default)"""

    def __init__(self, values, origin=None, frame=None, knots=None, target_mass=1.0):
        self.values = np.ascontiguousarray(np.asarray(values, dtype=np.float64))
        d = self.values.ndim
        self.nb_dims = d
        self.origin = np.zeros(d) if origin is None else np.asarray(origin, dtype=np.float64).reshape(d)
        if frame is None:
            step = np.ones(d)
        else:
            f = np.asarray(frame, dtype=np.float64)
            if f.ndim == 1:
                step = f.reshape(d)
            else:
                f = f.reshape(d, d)
                if np.count_nonzero(f - np.diag(np.diag(f))):
                    raise NotImplementedError("Image: only axis-aligned frames (a diagonal frame) are integrated here")
                step = np.diag(f).copy()
        if knots is not None:
            k = np.asarray(knots, dtype=np.float64).reshape(d, -1)
            for a in range(d):
                kk = k[a, : self.values.shape[a] + 1]
                if not np.allclose(np.diff(kk), kk[1] - kk[0]):
                    raise NotImplementedError("Image: only uniform knots are integrated here")
                self.origin[a] += kk[0] * step[a]
                step[a] *= kk[1] - kk[0]
        self.step = step
        self.target_mass = target_mass

    @property
    def mass(self):
        return float(self.values.sum() * np.prod(self.step))

    def normalized_version(self, nb_dims=None):
        if self.target_mass is None:
            return self
        m = self.mass
        if not m > 0:
            raise ValueError("Image: the values have no mass")
        res = Image.__new__(Image)
        res.values = self.values * (self.target_mass / m)
        res.nb_dims, res.origin, res.step, res.target_mass = self.nb_dims, self.origin, self.step, self.target_mass
        return res

    def box(self):
        return self.origin.copy(), self.origin + self.step * np.array(self.values.shape, dtype=np.float64)

    def bounding_half_spaces(self):
        lo, hi = self.box()
        d = self.nb_dims
        return np.concatenate([np.eye(d), -np.eye(d)]), np.concatenate([hi, -lo])

    def _sdot_density(self):
        if self.values.size == 1:
            lo, hi = self.box()
            return ("uniform", float(self.values.reshape(-1)[0]))
        if self.nb_dims != 2:
            raise NotImplementedError("Image: 3D images are not integrated by this build")
        return ("image", self.origin, self.step, self.values)


class SumOfGaussians(Distribution):
    """rho(x) = sum_i weights[i] exp(-|x - c_i|^2 / 2 s_i^2) / (2 pi s_i^2)^(d/2): `weights` are MASSES.
    The declared support is the box c_i +- support_sigmas s_i united (or `support_box`)."""

    def __init__(self, positions, sigmas, weights=None, target_mass=1.0, support_sigmas=6.0, support_box=None):
        self.positions = np.ascontiguousarray(np.asarray(positions, dtype=np.float64))
        self.nb_dims = self.positions.shape[1]
        self.sigmas = np.asarray(sigmas, dtype=np.float64).reshape(-1)
        self.weights = np.ones(len(self.sigmas)) if weights is None else np.asarray(weights, dtype=np.float64).reshape(-1)
        self.target_mass = target_mass
        self.support_sigmas = None if support_sigmas is None else float(support_sigmas)
        self.support_box = None if support_box is None else tuple(np.asarray(b, dtype=np.float64).reshape(-1) for b in support_box)

    @property
    def mass(self):
        return float(self.weights.sum())

    def normalized_version(self, nb_dims=None):
        if self.target_mass is None:
            return self
        return SumOfGaussians(self.positions, self.sigmas, self.weights * (self.target_mass / self.weights.sum()), self.target_mass,
                              self.support_sigmas, self.support_box)

    def box(self):
        if self.support_box is not None:
            return self.support_box[0].copy(), self.support_box[1].copy()
        if self.support_sigmas is None:
            return None
        k = self.support_sigmas
        return (self.positions - k * self.sigmas[:, None]).min(axis=0), (self.positions + k * self.sigmas[:, None]).max(axis=0)

    def bounding_half_spaces(self):
        b = self.box()
        if b is None:
            return None
        d = self.nb_dims
        return np.concatenate([np.eye(d), -np.eye(d)]), np.concatenate([b[1], -b[0]])

    def _sdot_density(self):
        return ("gauss", self.positions, self.sigmas, self.weights)


class Box:
    """a constant density on a box (an `Image` of one pixel once the dimension is known)"""

    def __init__(self, origin=None, frame=None, density=1.0, nb_dims=None):
        self.origin, self.frame, self.density = origin, frame, density
        d = nb_dims
        for a in (origin, frame):
            if a is not None:
                d = np.asarray(a).shape[0]
        self.nb_dims = d

    def image(self, nb_dims=None):
        d = self.nb_dims if self.nb_dims is not None else nb_dims
        if d is None:
            raise ValueError("Box: the dimension of the space is not known yet")
        origin = np.zeros(d) if self.origin is None else np.asarray(self.origin, dtype=np.float64).reshape(d)
        frame = np.eye(d) if self.frame is None else np.asarray(self.frame, dtype=np.float64)
        return Image(np.full((1,) * d, float(self.density)), origin=origin, frame=frame)

    def normalized_version(self, nb_dims=None):
        return self.image(nb_dims).normalized_version()

    def bounding_half_spaces(self):
        return self.image().bounding_half_spaces()
