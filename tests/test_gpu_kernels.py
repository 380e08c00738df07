"""Other kernels through the kernel seam (hfmm_b200.kernels, hfmm_plan_set_kernel_kind):
the screened-Coulomb (Yukawa) kernel exp(-kappa r)/(4 pi r) and its kappa = 0 case,
Laplace 1/(4 pi r), in every particle kernel, the device tables, the mixed near field
and the referee. Bars as for the Helmholtz path: potentials and fields to 1e-12 of
the oracle (kifmm.setup with the reference's yukawa / LAPLACE kernels, restated in
oracle/hfmm.py) and of the reference's own outputs (tests/golden/kernels/); the mixed
evaluate to 2e-6 of the FP64 one; the referee to 1e-13 of a NumPy direct sum."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from cases import uniform, clustered, sphere_clusters

pytestmark = pytest.mark.gpu
TOL = 1e-12
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "kernels", "*.npz")))


def _spec(kind, kappa):
    from hfmm_b200 import kernels
    return kernels.LAPLACE if kind == "laplace" else kernels.yukawa(kappa)


CASES = [
    ("yukawa_uniform", uniform, 3000, "yukawa", 3.0, 5, 24, None, "device"),
    ("yukawa_uniform_host", uniform, 3000, "yukawa", 3.0, 5, 24, None, "host"),
    ("yukawa_clustered", clustered, 2500, "yukawa", 8.0, 4, 16, None, "device"),
    ("laplace_sphere", sphere_clusters, 3000, "laplace", 0.0, 5, 20, None, "device"),
    ("laplace_depth4", uniform, 4000, "laplace", 0.0, 4, 16, 4, "device"),
]


@pytest.mark.parametrize("name,fn,n,kind,kappa,p,nmax,md,tables", CASES, ids=[c[0] for c in CASES])
def test_kernel_against_oracle(name, fn, n, kind, kappa, p, nmax, md, tables):
    import hfmm_b200
    pos, q = fn(n)
    q = np.real(q)
    spec = _spec(kind, kappa)
    st = hfmm_b200.kernel_setup(pos, spec, p=p, N_max=nmax, max_depth=md, tables=tables)
    ref = O.kernel_setup(pos, O.YukawaKernel(kappa), p=p, N_max=nmax, max_depth=md)
    assert st.info["max_depth"] == ref["max_depth"] and st.n_families == 1
    pot = hfmm_b200.kernel_evaluate(st, q)
    fld = hfmm_b200.kernel_evaluate(st, q, field=True)
    r_pot = np.asarray(O.evaluate_setup(ref, q)).reshape(-1)
    r_fld = np.asarray(O.evaluate_setup(ref, q, field=True)).reshape(-1, 3)
    assert O.relative_error(pot, r_pot) < TOL
    assert O.relative_error(fld, r_fld) < TOL
    # complex charges by linearity through evaluate_field
    q2 = q + 1j * np.cos(np.arange(n))
    phi, E = hfmm_b200.evaluate_field(st, q2)
    assert O.relative_error(phi.real, r_pot) < TOL
    assert O.relative_error(E.real, r_fld) < TOL
    st.close()


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_kernel_against_reference(path):
    import hfmm_b200
    with np.load(path) as z:
        g = {k: z[k] for k in z.files}
    spec = _spec(str(g["kind"]), float(g["kappa"]))
    st = hfmm_b200.kernel_setup(g["positions"], spec, p=int(g["p"]), N_max=int(g["N_max"]))
    assert st.info["max_depth"] == int(g["realised_depth"])
    pot = hfmm_b200.kernel_evaluate(st, g["charges"])
    fld = hfmm_b200.kernel_evaluate(st, g["charges"], field=True)
    assert O.relative_error(pot, g["pot"].reshape(-1)) < TOL
    assert O.relative_error(fld, g["field"].reshape(-1, 3)) < TOL
    st.close()


@pytest.mark.parametrize("kind,kappa", [("yukawa", 4.0), ("laplace", 0.0)])
def test_kernel_mixed_against_fp64(kind, kappa):
    import hfmm_b200
    pos, q = uniform(20000)
    st = hfmm_b200.kernel_setup(pos, _spec(kind, kappa), p=6, N_max=32, m2l_compress=1e-7)
    a = hfmm_b200.kernel_evaluate(st, q, field=True)
    b = hfmm_b200.kernel_evaluate(st, q, field=True, precision=hfmm_b200.PREC_MIXED)
    assert np.isfinite(b).all()
    assert O.relative_error(b, a) < 2e-6
    st.close()


def test_yukawa_referee():
    import hfmm_b200
    pos, q = uniform(3000)
    kappa = 2.5
    st = hfmm_b200.kernel_setup(pos, _spec("yukawa", kappa), p=4, N_max=16)
    tg = np.random.default_rng(4).choice(3000, 200, replace=False)
    phi, E = hfmm_b200.direct(st, q, tg, field=True)
    d = pos[tg][:, None, :] - pos[None, :, :]
    r = np.sqrt((d ** 2).sum(-1))
    ok = r > 0
    rs = np.where(ok, r, 1.0)
    G = np.where(ok, np.exp(-kappa * rs) / (4 * np.pi * rs), 0.0)
    W = np.where(ok, (1 + kappa * rs) * np.exp(-kappa * rs) / (4 * np.pi * rs ** 3), 0.0)
    assert O.relative_error(phi.real, G @ q) < 1e-13 and np.abs(phi.imag).max() == 0
    assert O.relative_error(E.real, np.einsum("ts,tsc,s->tc", W, d, q)) < 1e-13
    st.close()
