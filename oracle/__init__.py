"""CPU oracle for the TPFA hot path — TEST INFRASTRUCTURE ONLY.

A plain numpy/scipy restatement of the reference algorithms this package
accelerates, used only as the checker: by `tests/`, by
`__graft_entry__.smoke()` and by `bench.py`'s CPU-baseline leg.  Nothing in
`pymrst_b200/` imports it, and the product path never falls back to it.

Pinning: every function here is checked against golden fixtures generated by
running the reference itself (`tests/golden/make_golden.py`, which imports the
reference's Python package) and against the reference's MATLAB golden files
copied into the same fixtures.

Modules
-------
trans   compute_trans / harmonic face transmissibility
ow      two-phase oil-water fully-implicit residual, analytic Jacobian, wells,
        convergence, Newton step and schedule driver (direct solve)
incomp  incompressible TPFA pressure solve
"""
