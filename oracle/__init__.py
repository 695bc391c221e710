"""CPU oracle for the FL_correction hot path (test infrastructure only).

Nothing in ``fl_correction_b200`` imports this package.  It is loaded by the
tests, by ``__graft_entry__.smoke()`` and by the CPU-baseline legs of
``bench.py``, always as the checker or as the timed CPU reference, never as
part of the product path.
"""
