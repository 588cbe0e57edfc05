"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for molmot_b200.

The oracle restates the reference's FP64 algorithms on the CPU so that the
CUDA product path can be checked against them:

* ``oracle.rate_eq``  -- ctypes binding of ``rate_eq_oracle.c`` (1D force,
  batches over parameter sets, 1D Euler trajectories).
* ``oracle.force3d``  -- numpy restatement of the 3D rate-equation force and
  the 3D leapfrog integrator.
* ``oracle.flops``    -- algorithmic FLOP counts used for roofline figures.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its
``cpu_baseline`` leg and ``--impl reference``) may import this package, and
only as the checker or the timed CPU baseline.  The product package
``molmot_b200`` never imports it.
"""
