"""The CPU oracle: a NumPy restatement of solprop's reference arithmetic for the hot path.

This package is test infrastructure.  Only the tests, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import it, and only as the checker: nothing in
``solprop_b200`` calls it, and the product path fails loudly without its CUDA library.

Each function cites the reference file and line it restates (paths inside the solprop
repository).  The restatement is pinned: ``tests/test_oracle_golden.py`` checks it
against the golden vectors in ``tests/golden/``, which ``tests/golden/generate.py``
produced by running the reference's own ``numpy_ref`` backend on the same problems.
"""
