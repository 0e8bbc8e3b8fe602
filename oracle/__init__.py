"""CPU oracle for the SIFT + guided-matching path of PlaneSite (Edko01/FieldStitch).

TEST INFRASTRUCTURE ONLY. The modules here restate the reference's CPU algorithms
(app/planesite/gsift.py, features.py, matching.py) in NumPy/SciPy so that the CUDA path can be
checked against them. Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or as the timed CPU baseline; the
``fieldstitch_b200`` package never imports it and has no CPU fallback.

Pinning: ``tests/golden/make_golden.py`` runs the reference itself (imported from its source tree
in the build container) on seeded inputs and stores the outputs under ``tests/golden/``;
``tests/test_oracle_golden.py`` checks these modules against them.
"""
