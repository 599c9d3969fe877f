"""Oracle package: TEST INFRASTRUCTURE ONLY.

Nothing in the product (the ``yasf_b200`` package) imports, links or executes
anything under this directory. Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` use it, and only as the parity reference or as
the timed CPU baseline.

Contents
--------
``stubs/``        stand-in modules that let the upstream ``yasfpy`` package import in
                  a container that lacks its third-party dependencies
                  (``pywigxjpf``, ``refidxdb``, ``pyperf``). Used only by
                  ``tests/golden/make_golden.py`` to generate golden fixtures.
``cpu_ref.c``     a plain-C (OpenMP) restatement of the reference's CPU coupling
                  kernel ``particle_interaction_scalar`` (yasfpy/functions/cpu_numba.py:22-95),
                  its pairwise lookups (yasfpy/functions/misc.py:117-243,
                  yasfpy/functions/legendre_normalized_trigon.py:12-95) and the
                  scattering cross section (yasfpy/functions/cpu_numba.py:410-457).
``restate.py``    numpy restatements of the setup arithmetic (translation table,
                  Mie coefficients, plane-wave coefficients, SciPy-semantics GMRES)
                  plus ctypes access to ``cpu_ref.c``.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every function here against
fixtures generated by running the upstream reference itself
(``tests/golden/make_golden.py``) and against the MATLAB/CELES golden vectors that the
reference's own tests hold (converted to ``tests/golden/celes_*.npz``).
"""
