"""Oracle: CPU restatement of the reference's algorithms, for TESTS ONLY.

This package is test infrastructure.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import it, and only as the checker
(or the timed CPU baseline), never as the thing measured or shipped.  The
product (``evd4sc2025_b200``) never imports it and has no CPU fallback.

Each function cites the reference file:line it restates (paths relative to the
hansheng1001/EVD4SC2025 source tree).  The reference ships no tests, golden
vectors or fixtures; the restatement is pinned by (1) LAPACK (scipy) on the
same inputs through exact invariants (spectrum preserved by every similarity
stage, orthogonality of every factor), and (2) outputs of the reference's own
GPU build run on a B200 (``oracle/ref_driver.cu`` via ``oracle/Makefile``),
stored as fixtures under ``tests/golden/``.
"""
