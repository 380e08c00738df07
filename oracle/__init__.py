"""CPU oracle for the Helmholtz KIFMM evaluate path (test infrastructure only).

This package is a NumPy restatement of the reference's HFMM path (HFMM.py,
jaxfmm/kifmm/*, jaxfmm/core.py, jaxfmm/near.py, jaxfmm/trees/*). It exists to
check the CUDA product: only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it, and never as the thing that is
measured or shipped.

Pinning: the reference ships no golden vectors and JAX is not installed here,
so the reference's own Python code was run on a NumPy stand-in for the JAX calls
it makes (tests/golden/jax_on_numpy.py, tests/golden/make_golden.py) and its
outputs committed as fixtures: standard and edge cases (tests/golden/*.npz,
tests/golden/edge/), the 2e4-point CPU-runnable configuration (tests/golden/c1/),
the reference's test.py grid (tests/golden/grid/) and per-phase outputs
(tests/golden/phases/). The oracle matches them bit for bit on every integer
array (tree, sort order, particles-in-leaf, U/V/W/X/near lists, buffer sizes),
phase by phase through the potential each density makes on its check surface,
and to the rounding floor on potentials and fields (tests/test_golden.py,
tests/test_oracle_known_answers.py). It also passes the reference's known-answer
checks (test.py:63-72) and an O(N^2) direct sum.
"""

from .surfaces import n_surf, surface_pts, R_EQUIV, R_CHECK
from .operators import (helmholtz_G_np, pinv_factors, build_operators,
                        build_operators_leveled)
from .tree import (morton_encode, morton_decode, build_fmm_tree, build_fmm_tree_auto,
                   assign_particles, box_geometry, NEIGH_OFFSETS, ADJ_CHILD_MASK)
from .lists import build_v, build_u, build_wx, near_pairs
from .hfmm import (setup, evaluate, evaluate_setup, evaluate_complex, kifmm_setup,
                   direct, direct_field, relative_error, YukawaKernel, kernel_setup)

__all__ = [
    "n_surf", "surface_pts", "R_EQUIV", "R_CHECK",
    "helmholtz_G_np", "pinv_factors", "build_operators", "build_operators_leveled",
    "morton_encode", "morton_decode", "build_fmm_tree", "build_fmm_tree_auto",
    "assign_particles", "box_geometry", "NEIGH_OFFSETS", "ADJ_CHILD_MASK",
    "build_v", "build_u", "build_wx", "near_pairs",
    "setup", "evaluate", "evaluate_setup", "evaluate_complex", "kifmm_setup",
    "direct", "direct_field", "relative_error", "YukawaKernel", "kernel_setup",
]
