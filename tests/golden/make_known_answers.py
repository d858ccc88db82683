"""Writes known_answers.json: the reference's own known-answer tests for the power-diagram path, restated as
(input, expected) fixtures.  The expected values are the analytic answers those tests assert; nothing here
runs the reference (it cannot be imported here: it needs the absent third-party `loom`).

    python tests/golden/make_known_answers.py

Each case cites the test it restates (paths relative to the reference project).
"""
import json
import os

import numpy as np

cases = []

# tests/test_PowerDiagram.py:35-44 -- two symmetric seeds in the unit square: each takes half
cases.append(dict(name="basic_2D", src="tests/test_PowerDiagram.py:35-44", positions=[[0.25, 0.5], [0.75, 0.5]], weights=None,
                  lo=[0, 0], hi=[1, 1], masses=[0.5, 0.5], atol=1e-12))

# tests/test_PowerDiagram.py:46-56 -- one seed takes the whole box, 2^d (d = 2, 3)
for d in (2, 3):
    cases.append(dict(name=f"one_seed_takes_everything_{d}d", src="tests/test_PowerDiagram.py:46-56", positions=[[0.3] * d], weights=None,
                      lo=[0] * d, hi=[2.0] * d, masses=[2.0 ** d], atol=1e-12))

# tests/test_PowerDiagram.py:217-231 -- a regular 3 x 3 grid: every square is 1/9
xs = [1 / 6, 3 / 6, 5 / 6]
cases.append(dict(name="seeds_on_a_grid", src="tests/test_PowerDiagram.py:217-231", positions=[[x, y] for x in xs for y in xs], weights=None,
                  lo=[0, 0], hi=[1, 1], masses=[1 / 9] * 9, atol=1e-12))

# tests/test_PowerDiagram.py:233-243 -- a 2 x 2 x 2 grid: every cube is 1/8
xs = [0.25, 0.75]
cases.append(dict(name="seeds_on_a_3D_grid", src="tests/test_PowerDiagram.py:233-243", positions=[[x, y, z] for x in xs for y in xs for z in xs],
                  weights=None, lo=[0, 0, 0], hi=[1, 1, 1], masses=[1 / 8] * 8, atol=1e-12))

# tests/test_PowerDiagram.py:245-264 -- a seed outside the domain has an empty cell; the others still tile it
cases.append(dict(name="a_seed_outside_the_domain_has_no_cell", src="tests/test_PowerDiagram.py:245-264",
                  positions=[[0.5, 0.5], [0.2, 0.2], [5.0, 5.0]], weights=None, lo=[0, 0], hi=[1, 1], masses=None,
                  mass_at={"2": 0.0}, total=1.0, atol=1e-12))

# tests/test_PowerDiagram.py:266-284 -- the bisector is shifted by the weight gap: the left cell measures (1 + gap) / 2
for gap in (-0.6, -0.25, 0.0, 0.25, 0.6):
    cases.append(dict(name=f"the_bisector_is_shifted_by_the_weight_gap_{gap}", src="tests/test_PowerDiagram.py:266-284",
                      positions=[[0.0, 0.5], [1.0, 0.5]], weights=[gap, 0.0], lo=[0, 0], hi=[1, 1], masses=[(1 + gap) / 2, (1 - gap) / 2],
                      atol=1e-12))

# tests/test_PowerDiagram.py:374-388 -- a dominated seed loses its cell
cases.append(dict(name="a_dominated_seed_loses_its_cell", src="tests/test_PowerDiagram.py:374-388",
                  positions=[[0.25, 0.5], [0.5, 0.5], [0.75, 0.5]], weights=[0.0, -1.0, 0.0], lo=[0, 0], hi=[1, 1], masses=None,
                  mass_at={"1": 0.0}, total=1.0, atol=1e-12))

# tests/test_PowerDiagram.py:390-403 -- a big enough weight swallows the domain
cases.append(dict(name="a_big_enough_weight_swallows_the_domain", src="tests/test_PowerDiagram.py:390-403",
                  positions=[[0.25, 0.4], [0.5, 0.6], [0.8, 0.3]], weights=[0.0, 10.0, 0.0], lo=[0, 0], hi=[1, 1], masses=[0.0, 1.0, 0.0],
                  atol=1e-12))

# tests/test_PowerDiagram.py:111-125 -- an off-centre box: the cells tile its volume
rng = np.random.default_rng(7)
mi, ma = np.array([-2.0, 1.0, 0.5]), np.array([1.0, 4.0, 2.5])
pos = rng.uniform(mi + 0.1, ma - 0.1, size=(15, 3))
cases.append(dict(name="an_off_centre_box", src="tests/test_PowerDiagram.py:111-125", positions=pos.tolist(), weights=None, lo=mi.tolist(),
                  hi=ma.tolist(), masses=None, total=float(np.prod(ma - mi)), atol=1e-10))

# tests/test_PowerDiagram.py:58-75 and 322-337 -- the cells tile the unit box, with and without weights (d = 2, 3)
for d, n in ((2, 60), (3, 40)):
    rng = np.random.default_rng(12 + d)
    pos = rng.uniform(0.05, 0.95, size=(n, d))
    cases.append(dict(name=f"sum_is_the_domain_{d}d", src="tests/test_PowerDiagram.py:58-75", positions=pos.tolist(), weights=None,
                      lo=[0] * d, hi=[1] * d, masses=None, total=1.0, positive=True, atol=1e-10))
for d, n in ((2, 40), (3, 25)):
    rng = np.random.default_rng(50 + d)
    pos = rng.uniform(0.05, 0.95, size=(n, d))
    w = rng.uniform(-0.1, 0.1, size=n)
    cases.append(dict(name=f"weighted_cells_still_tile_the_domain_{d}d", src="tests/test_PowerDiagram.py:322-337", positions=pos.tolist(),
                      weights=w.tolist(), lo=[0] * d, hi=[1] * d, masses=None, total=1.0, atol=1e-10))

here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "known_answers.json"), "w") as f:
    json.dump(cases, f, indent=1)
print(len(cases), "cases")
