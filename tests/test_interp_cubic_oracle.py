"""The cubic g0 interpolation of the oracle (an extension: keldy interpolates linearly):
exact on cubic polynomials, including the two ends of the mesh, and far more accurate
than linear interpolation on the flat-band table away from t = 0."""
import numpy as np

from keldy_b200 import g0_tables


def _g0(oracle, model, t):
    return np.array([oracle.g0(model, (x, 0, 0, 0, 0), (0.0, 0, 0, 0, 0)) for x in t])


def test_cubic_reproduces_cubics(oracle):
    t = g0_tables.time_mesh(2.0, 41)
    p = lambda x: (0.3 - 0.1j) + (0.5 + 2j) * x - 0.7 * x ** 2 + (0.25 - 0.5j) * x ** 3  # noqa: E731
    m = oracle.model(2.0, p(t), p(t), interp=3)
    x = np.concatenate([np.linspace(-2.0, 2.0, 97), [-2.0, -1.99, 1.99, 2.0]])
    got = _g0(oracle, m, x)
    # (x, 0) is later than (0, 0) on the forward branch for x > 0 (g^>), earlier for x < 0 (g^<)
    np.testing.assert_allclose(got, p(x), rtol=0, atol=1e-12)
    lin = oracle.model(2.0, p(t), p(t))
    assert np.abs(_g0(oracle, lin, x) - p(x)).max() > 1e-3


def test_cubic_accuracy_on_flatband(oracle):
    _, le, gr = g0_tables.flatband(1.0, 0.3, 0.4, 20.0, 10.0, 2001)
    tf, lf, gf = g0_tables.flatband(1.0, 0.3, 0.4, 20.0, 10.0, 8001)  # mesh 4x finer: the quarter points
    lin = oracle.model(10.0, le, gr)
    cub = oracle.model(10.0, le, gr, interp=3)
    sel = np.where((np.arange(len(tf)) % 4 != 0) & (np.abs(tf) > 0.5))[0][::37]
    want = np.where(tf[sel] > 0, gf[sel], lf[sel])
    e_lin = np.abs(_g0(oracle, lin, tf[sel]) - want).max()
    e_cub = np.abs(_g0(oracle, cub, tf[sel]) - want).max()
    assert e_cub < 1e-3 * e_lin, (e_cub, e_lin)
