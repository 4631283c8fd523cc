"""CPU oracle for the statevector tile executor.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` as the checker / the timed CPU baseline.  Nothing in
``frontierlabproject_b200`` imports it, and the product path has no CPU fallback.

* ``statevector.py`` -- numpy restatement of the reference's per-gate kernels, permute
  semantics, fusion and tile loop, plus an FP64 adjoint gradient.
* ``cpu_kernels.c``  -- the same per-gate arithmetic in C with OpenMP, timed as the CPU
  baseline; built by ``oracle/build.py`` into ``oracle/libqsim_oracle.so``.
"""
