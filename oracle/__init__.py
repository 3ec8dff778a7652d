"""CPU oracle for the forced pseudospectral DNS step with droplets.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this directory; only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` use it, and only to check the GPU results or as the timed CPU baseline.

Contents (FP64, NumPy/SciPy, numba for the droplet loops):
  * ``reference_np`` - a restatement of the reference's own single-rank algorithm
    (forced-dns-sm.py + particles.py): grid operators, slab transforms, forcing, full RHS, RK4
    time loop, cosine-kernel droplet gather/deposition, droplet RHS;
  * ``config_np``    - the semantics of the benchmark configurations that the reference does not
    have (RK2 with viscous integrating factor, shells |k|<=2 constant-power forcing, trilinear /
    tricubic gather, Stokes drag + settling droplets with Heun);
  * ``collide_np``   - cell-list collision pairs (bit-exact FP64 rule);
  * ``exact_np``     - direct Fourier-sum velocity at points;
  * ``mlp_np``       - the learned-interpolation MLP forward/backward in FP32/FP64.

Parity pin: ``reference_np`` is checked against golden vectors that were produced by running the
reference scripts themselves (tests/golden/make_golden.py, fixtures ``tests/golden/ref_*.npz``).
"""
