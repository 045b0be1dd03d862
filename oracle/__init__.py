"""CPU oracle for the graph-state scan engine -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain Python/NumPy, the reference algorithms that the
CUDA engine replaces (whyihaveyou/rgs70-classical-challenge, paths relative to
that project, ``W/`` = ``work/rgs_attack/``):

* ``scan_plan``   -- the GF(2) scan compiler and the NumPy sweep executor
                     (``W/upstream_scan/scan_plan.py``);
* ``graph_state`` -- statevector, conditional-state and Fourier-covariant
                     helpers (``W/graph_sampler.py``,
                     ``W/fourier_covariant_sampler.py``,
                     ``W/deferred_global_sampler.py``,
                     ``W/init_specialization.py``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this package, and only as
the checker or as the timed CPU baseline.  The product path (the package next
to this directory) never imports it: it fails loudly when its CUDA library is
missing instead of falling back to this code.

Parity pin: every function here is checked against fixtures generated by
importing the reference itself (``tests/golden/make_golden.py``) and against the
reference's own stored complex128 records of the RGS70 instance.
"""
