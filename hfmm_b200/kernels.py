"""Kernel specifications of the kernel seam (the reference's ``Kernel`` NamedTuple,
jaxfmm/kernels/spec.py:10-62, with its Laplace and Yukawa kernels,
kernels/laplace/kernel.py:104 and kernels/yukawa/kernel.py:10-75).

The reference passes callables (host matrix, device value, gradient, near-field
weights) for XLA to trace; here the device evaluates the kernels itself, so a
specification names the kernel the CUDA path computes (``hfmm_plan_set_kernel_kind``)
and its parameter:

* ``helmholtz(k)``: the two components cos(kr)/r and sin(kr)/r of HFMM.py:12-52
  (one family when k = 0);
* ``yukawa(kappa)``: exp(-kappa r) / (4 pi r), one family;
* ``LAPLACE``: 1 / (4 pi r), the screened kernel at kappa = 0.
"""
from typing import NamedTuple

import numpy as np

__all__ = ["KernelSpec", "helmholtz", "yukawa", "LAPLACE"]


class KernelSpec(NamedTuple):
    name: str
    kind: str          # "helmholtz" or "yukawa"
    param: float       # k, or kappa
    families: int      # kernel families the plan evaluates (2 for Helmholtz with k != 0)


def helmholtz(k):
    k = float(k)
    if not np.isfinite(k):
        raise ValueError("k must be a finite real number")
    return KernelSpec(f"helmholtz({k:g})", "helmholtz", k, 1 if k == 0 else 2)


def yukawa(kappa):
    kappa = float(kappa)
    if not (np.isfinite(kappa) and kappa >= 0):
        raise ValueError("kappa must be a finite number >= 0")
    return KernelSpec(f"yukawa(kappa={kappa:g})", "yukawa", kappa, 1)


LAPLACE = KernelSpec("laplace", "yukawa", 0.0, 1)
