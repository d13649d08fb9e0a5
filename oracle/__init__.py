"""CPU FP64 oracle for the structural hot path of EXFEM (package ``gfem`` 0.3.0).

TEST INFRASTRUCTURE ONLY.  This package is a line-by-line CPU restatement of the
reference's element, material, assembly and linear-solver arithmetic.  It exists
to check the CUDA product path; it is never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it, and there only as the checker (or as the timed CPU reference arm).  The
``exfem_b200`` package never imports it and has no CPU fallback.

Why a restatement: the reference is Python on JAX/XLA (``gfem/__init__.py:14``
imports jax) and JAX and PyAMG are not installable here, so the reference cannot
run.  Tangents are still obtained by automatic differentiation (``torch.func``
jacfwd / vjp / jvp on CPU FP64), exactly as the reference obtains them with
``jax.jacfwd`` / ``jax.vjp`` / ``jax.jvp``.

How it is pinned (no golden vectors exist in the reference, ``tests/`` holds
only analytic checks and cross-solver agreement):

* the reference's own known-answer tests, re-run on the oracle:
  patch tests (tests/test_verification.py:27-36), J2 uniaxial hardening vs the
  closed form (tests/test_verification.py:39-52), TET10 cantilever vs
  Timoshenko beam theory and reaction balance (tests/test_verification.py:66-83),
  iterative-vs-direct agreement (tests/test_gpu_paths.py:47-55);
* mesh fixtures generated by importing the reference's pure-NumPy
  ``gfem/mesh.py`` by file path (``tests/golden/make_golden.py``);
* finite-difference checks of every AD tangent.

The smoothed-aggregation hierarchy (PyAMG in the reference) is parity unpinned:
no reference test pins it and PyAMG is absent.  The oracle therefore checks the
V-cycle *application* on a given hierarchy, and checks converged solutions
against a sparse direct solve.

Modules: ``fem`` (elements, materials, element kernels, index maps, global
operators), ``linalg`` (PCG, CSR helpers, rigid-body modes, Chebyshev V-cycle,
direct solve), ``solvers`` (load/BC set-up, Newton with line search and
automatic incrementation), ``loads`` (surface skin and pressure vectors).
"""
