"""CPU checks of the oracle: analytic pins and the committed golden fixtures."""
import glob
import os

import numpy as np
import pytest

from gitm_b200 import abi, synthetic

HERE = os.path.dirname(os.path.abspath(__file__))


def test_limiter_mc_truth_table(oracle_lib):
    L = oracle_lib.limiter_mc
    # same sign: min of beta*u, beta*d, mean (ModLimiter.f90:73-76)
    assert L(1.0, 3.0, 2.0) == 2.0
    assert L(1.0, 1.5, 2.0) == 1.25
    assert L(3.0, 1.0, 1.0) == 1.0
    assert L(-1.0, -3.0, 2.0) == -2.0
    assert L(-3.0, -1.0, 1.0) == -1.0
    # opposite signs or a zero slope: 0
    for u, d in [(1.0, -1.0), (-1.0, 1.0), (0.0, 1.0), (1.0, 0.0), (0.0, -1.0), (-2.0, 0.0), (0.0, 0.0)]:
        assert L(u, d, 2.0) == 0.0


def test_lu_matches_numpy(oracle_lib):
    rng = np.random.default_rng(5)
    for _ in range(50):
        a = rng.normal(size=(6, 6)) + 6 * np.eye(6)
        b = rng.normal(size=6)
        x, ok = oracle_lib.lu_solve(a, b)
        assert ok
        np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=1e-12, atol=1e-13)
    # a row of zeros is the stop_gitm('singular matrix in ludcmp') case
    a = rng.normal(size=(6, 6))
    a[3] = 0.0
    _, ok = oracle_lib.lu_solve(a, np.ones(6))
    assert not ok


@pytest.mark.parametrize("n_alts", [20, 50, 100])
def test_mesh_coefficients_exact_for_quartics(oracle_lib, n_alts):
    alt = synthetic.make_altitude_grid(n_alts)
    grad, low, up = oracle_lib.mesh_coefs(alt)
    z = (alt - alt[2]) / 1e5
    rng = np.random.default_rng(n_alts)
    p = rng.normal(size=5)
    f = np.polyval(p, z)
    df = np.polyval(np.polyder(p), z) / 1e5
    g = lambda i: i + 1  # noqa: E731  Fortran cell -> index
    for i in range(1, n_alts + 1):  # centred 5-point stencil (vertical_solver_rusanov.f90:511-543)
        est = sum(grad[i - 1, k] * f[g(i - 2 + k)] for k in range(5))
        assert est == pytest.approx(df[g(i)], rel=1e-7, abs=1e-12)
    for k, i in enumerate((0, -1)):  # forward derivative at cell i+1 (set_vertical_bcs.Earth.f90:279-297)
        est = sum(low[k, j] * f[g(i + 1 + j)] for j in range(5))
        assert est == pytest.approx(df[g(i + 1)], rel=1e-7, abs=1e-12)
    for k, i in enumerate((n_alts + 1, n_alts + 2)):  # backward derivative at cell i-1 (:505-525)
        est = sum(up[k, j] * f[g(i - 1 - j)] for j in range(5))
        assert est == pytest.approx(df[g(i - 1)], rel=1e-7, abs=1e-12)


GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load_golden(path):
    from tests.golden.make_golden import CASES

    d = np.load(path)
    name = os.path.basename(path)[:-4]
    n_cols, n_alts, seed, n_steps, dt, over, mkw = CASES[name]
    p = abi.default_params(**over)
    fields = {k[3:]: d[k] for k in d.files if k.startswith("in_")}
    m = synthetic.Member(n_alts=int(d["n_alts"]), n_cols=int(d["n_cols"]),
                         **{k: v.copy() for k, v in fields.items()})
    out = {k[4:]: d[k] for k in d.files if k.startswith("out_")}
    return p, m, out, int(d["n_steps"]), float(d["dt"]), d["status"]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_reproduces_golden(oracle_lib, path):
    p, m, out, n_steps, dt, status = load_golden(path)
    st = oracle_lib.advance(m, p, dt, n_steps, nthreads=2)
    np.testing.assert_array_equal(st, status)
    for k in synthetic.Member.STATE + ("log_ns", "ndensity"):
        np.testing.assert_allclose(getattr(m, k), out[k], rtol=1e-14, atol=0, err_msg=k)


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 5


def test_oracle_columns_independent(oracle_lib):
    """Advancing columns together or one at a time gives identical results."""
    p = abi.default_params()
    m = synthetic.make_member(5, 30, seed=3)
    whole = m.copy()
    oracle_lib.advance(whole, p, 2.0, 2, nthreads=3)
    from gitm_b200.parallel import shard_member
    for r in range(5):
        part = shard_member(m, r, 5)
        oracle_lib.advance(part, p, 2.0, 2, nthreads=1)
        for k in synthetic.Member.STATE:
            np.testing.assert_array_equal(getattr(part, k), getattr(whole, k)[..., r:r + 1])


def test_oracle_neg_density_stops_column(oracle_lib):
    p = abi.default_params()
    m = synthetic.make_member(4, 20, seed=4)
    m.ndensity_s[2, 10, 1] = 0.0  # column 1 has a non-positive density
    before = m.copy()
    st = oracle_lib.advance(m, p, 2.0, 1)
    assert st[1] & abi.ST_NEG_DENSITY and st[0] == 0 and st[2] == 0
    for k in synthetic.Member.STATE:
        np.testing.assert_array_equal(getattr(m, k)[..., 1], getattr(before, k)[..., 1])


def test_operation_count(oracle_lib):
    p = abi.default_params()
    m = synthetic.make_member(1, 50, seed=1)
    d = synthetic.to_modvertical(m, p)
    ops = oracle_lib.count_ops(d, p, 2.0)
    flops = ops["add"] + ops["mul"] + ops["div"] + ops["sqrt"] + 20 * ops["trans"]
    # a few hundred thousand flop-equivalents per column-step
    assert 2e5 < flops < 2e6, ops


def test_oracle_heating_update(oracle_lib):
    """add_sources' temperature line: interior cells gain dt * scale * heating."""
    from gitm_b200 import abi, synthetic
    m = synthetic.make_member(8, 50, seed=3, with_heating=True)
    m0 = synthetic.make_member(8, 50, seed=3)
    p = abi.default_params()
    a, b = m.copy(), m0.copy()
    oracle_lib.advance(a, p, 2.0, 1)
    oracle_lib.advance(b, p, 2.0, 1)
    d = a.temperature - b.temperature
    want = 2.0 * (m.heating_scale[None, None, :] * m.heating)
    # the difference of two temperatures: exact to a few ulps of T
    np.testing.assert_allclose(d[0, 2:-2], want[0, 2:-2], rtol=1e-9,
                               atol=4e-16 * np.abs(b.temperature).max())
    assert np.abs(d[0, [0, 1, -2, -1]]).max() == 0.0


def _eddy_profile(pressure, p):
    """calc_eddy_diffusion_coefficient (Earth.f90:376-411), numpy form."""
    k = np.zeros_like(pressure)
    taper = p.eddy_coef * (pressure - p.eddy_pressure1) / (p.eddy_pressure0 - p.eddy_pressure1)
    k = np.where(pressure > p.eddy_pressure1, taper, k)
    return np.where(pressure > p.eddy_pressure0, p.eddy_coef, k)


def test_oracle_eddy_producer(oracle_lib):
    """compute_eddy: after a step, KappaEddyDiffusion(1:nAlts) is the profile
    of Pressure = Temperature * Rho at the start of that step; the step itself
    reads the coefficient passed in, the next step the produced one."""
    from gitm_b200 import abi, synthetic
    m = synthetic.make_member(16, 50, seed=8, with_heating=True)
    p = abi.default_params(compute_eddy=1)
    p0 = abi.default_params()
    pressure = m.temperature * m.rho
    want = _eddy_profile(pressure, p)
    # the synthetic columns cover all three regimes of the profile
    inner = pressure[0, 2:-2]
    assert (inner > p.eddy_pressure0).any() and (inner <= p.eddy_pressure1).any()
    assert ((inner > p.eddy_pressure1) & (inner <= p.eddy_pressure0)).any()
    a, b = m.copy(), m.copy()
    oracle_lib.advance(a, p, 2.0, 1)
    oracle_lib.advance(b, p0, 2.0, 1)
    for k in synthetic.Member.STATE:
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    np.testing.assert_array_equal(a.eddy[0, 2:-2], want[0, 2:-2])
    np.testing.assert_array_equal(a.eddy[0, [0, 1, -2, -1]], m.eddy[0, [0, 1, -2, -1]])
    # two steps = one step, the produced coefficient, one more step
    two = m.copy()
    oracle_lib.advance(two, p, 2.0, 2)
    c = b.copy()
    c.eddy[0, 2:-2] = want[0, 2:-2]
    p1 = c.temperature * c.rho
    oracle_lib.advance(c, p0, 2.0, 1)
    for k in synthetic.Member.STATE:
        np.testing.assert_array_equal(getattr(two, k), getattr(c, k), err_msg=k)
    np.testing.assert_array_equal(two.eddy[0, 2:-2], _eddy_profile(p1, p)[0, 2:-2])
