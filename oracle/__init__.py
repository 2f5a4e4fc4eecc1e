"""CPU oracle for the TUPS parquet-loop hot path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The
product path (``tups_b200``) never imports it.
"""
