"""The oracle: CPU restatement and the reference's own FP64 force path.

Test infrastructure.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
bench's CPU-baseline leg load anything from here, as the reference results
to compare with; the engine never does.
"""
