"""CPU restatement of the reference solver (TEST INFRASTRUCTURE ONLY).

Nothing in the product package imports this directory.  It is used by
``tests/``, by ``__graft_entry__.smoke()`` as the checker and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.

The reference (BMOLKAIST/Inverse_solver) is MATLAB code that cannot run in
this environment, and it ships no golden vectors, so parity is *unpinned*:
the restatement follows the reference line by line (citations in each
docstring) and is pinned only by the known-answer properties the reference
itself provides (Hankel transform vs the analytic J1 transform,
``hankel_transform/test_hankel.m``; zero residues after unwrapping,
``goldstein_GPU/show_unwrapping_performance.m``) plus physics identities.
"""
