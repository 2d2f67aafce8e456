"""CPU oracle for the B200 Ros2 path: a NumPy/SciPy FP64 restatement of the
reference VULCAN-JAX functions on the hot path.

TEST INFRASTRUCTURE ONLY. Imported solely by ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline / reference
leg), always as the checker or the timed CPU baseline and never as the product.
Pinned against the reference's own code run in the build container through a
NumPy stand-in for JAX (fixtures in ``tests/golden/``, made by
``tests/golden/make_golden.py``).
"""
