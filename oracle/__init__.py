"""CPU oracle for the GPU hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU, the reference algorithms of the path the GPU kernels
implement, so that tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` can check and time against them.  The product (``concrete_impact_b200``)
never imports it.

* ``oracle.j2vp``       -- NumPy restatement of the J2 Perzyna return map
                          (src/fem/materials/plasticity.py of the reference).
* ``oracle.j2vp_loop``  -- the same algorithm as a per-point loop, mirroring the
                          reference's own per-point execution (used to time the
                          reference's CPU cost where the reference itself cannot run).
* ``oracle/j2vp_oracle.c`` -- plain-C restatement of the batched incremental form,
                          multi-threaded with OpenMP, used as the strong CPU baseline.
* ``oracle.rve``        -- NumPy/SciPy restatement of the periodic Hex8 RVE Newton solve;
  ``oracle.rve_general`` -- the same on any mesh with topology-provided periodic classes.
* ``oracle.fe2``        -- explicit macro dynamics of a linear elastic bar.
* ``oracle.newmark``    -- implicit Newmark material dynamics (the reference's
                          solve_material_implicit_newmark) with J2 points or RVE solves.
* ``oracle.rno`` / ``oracle.rno_torch`` -- the package's recurrent surrogate window and a
                          host torch training loop (CPU baseline).
* ``oracle.rno_energy`` -- the reference's energy-based RVE-RNO update.

Parity pin: every function is checked against golden vectors produced by running the
reference implementation itself (``tests/golden/make_golden.py``) and against the
reference's own closed-form and finite-difference tests (``tests/test_oracle.py``).
"""
