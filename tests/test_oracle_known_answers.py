"""The reference's own known-answer checks (test.py:24-77) run against the oracle.

The reference ships no golden vectors; its test.py assertions are its known
answers, and on its default grid the oracle's potentials also equal the
reference's own (tests/golden/grid/, made by running the reference's code, see
tests/golden/make_golden.py): complex128 finite output, relative
L2 error vs the O(N^2) direct sum below 5e-2 (p <= 3) or 5e-3 (p > 3) for the
total, real and imaginary parts, linearity at 1e-10, an exactly-zero imaginary
part at k = 0, and errors that improve with p against the smallest p.
"""
import numpy as np
import pytest

import os

import oracle as O
from cases import uniform, clustered

# The reference's own potentials on this grid: tests/golden/make_golden.py --grid ran
# its test.py checks on them (they pass) and stored them.
GRID = os.path.join(os.path.dirname(__file__), "golden", "grid", "test_py_grid.npz")


@pytest.mark.parametrize("n", [256, 640])
@pytest.mark.parametrize("clust", [False, True])
def test_reference_grid(n, clust):
    pos, q = (clustered if clust else uniform)(n)
    with np.load(GRID) as z:
        tag = f"{'clustered' if clust else 'uniform'}{n}"
        grid = {key: z[key] for key in z.files if key.startswith(tag + "_")}
    assert np.array_equal(grid[tag + "_positions"], pos) and np.array_equal(grid[tag + "_charges"], q)
    for k in (0.0, 1.0, 3.0):
        ref = O.direct(pos, q, k)
        baseline = None
        for p in (3, 5):
            st = O.setup(pos, k, p=p, N_max=16)
            act = O.evaluate(st, q)
            assert act.dtype == np.complex128 and np.isfinite(act).all()
            # the reference's own output on the same case, to its rounding floor
            assert O.relative_error(act, grid[f"{tag}_k{k:g}_p{p}_phi"]) < 1e-12
            errs = np.array([O.relative_error(a, b) for a, b in
                             ((act, ref), (act.real, ref.real), (act.imag, ref.imag))])
            # the same errors; an error near 1e-11 (the sin part at k = 1) moves by the
            # rounding floor of the potential, so the bar has an absolute part
            np.testing.assert_allclose(errs, grid[f"{tag}_k{k:g}_p{p}_errors"], rtol=1e-6, atol=1e-12)
            assert max(errs) < (5e-2 if p <= 3 else 5e-3), errs
            np.testing.assert_allclose(O.evaluate(st, -0.5 * q), -0.5 * act, rtol=1e-10, atol=1e-10)
            if k == 0:
                assert np.count_nonzero(act.imag) == 0
            if baseline is not None:
                assert np.all(errs < np.maximum(0.8 * baseline, 2e-6)), errs
            baseline = errs if baseline is None else baseline


def test_evaluate_rejects_complex_and_bad_shape():
    pos, q = uniform(64)
    st = O.setup(pos, 1.0, p=3, N_max=16)
    with pytest.raises(ValueError):
        O.evaluate(st, q + 1j)
    with pytest.raises(ValueError):
        O.evaluate(st, q[:-1])


@pytest.mark.parametrize("bad", [
    dict(positions=np.zeros((0, 3))), dict(positions=np.zeros((4, 2))),
    dict(positions=np.array([[0.0, 0.0, np.nan]])), dict(p=1), dict(p=2.5),
    dict(N_max=0), dict(max_depth=0), dict(k=np.inf)])
def test_setup_validation(bad):
    args = dict(positions=uniform(32)[0], k=1.0, p=3, N_max=16, max_depth=None)
    args.update(bad)
    with pytest.raises(ValueError):
        O.setup(**args)


def test_complex_and_field_against_direct():
    from cases import complex_uniform
    pos, q = complex_uniform(800)
    k = 2.0
    st = O.setup(pos, k, p=5, N_max=32)
    phi, E = O.evaluate_complex(st, q, field=True)
    assert O.relative_error(phi, O.direct(pos, q, k)) < 5e-3
    assert O.relative_error(E, O.direct_field(pos, q, k)) < 5e-3
    # linearity with complex charges equals the real evaluate combination
    re = O.evaluate(st, q.real)
    im = O.evaluate(st, q.imag)
    np.testing.assert_allclose(phi, re + 1j * im, rtol=1e-11, atol=1e-11)
