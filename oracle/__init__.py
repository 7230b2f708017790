"""TEST INFRASTRUCTURE ONLY: the CPU oracle (compiled reference + C restatement).

Imported by tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` only.
"""
