"""CPU oracle for the channel3D RK3 fractional-step path -- TEST INFRASTRUCTURE ONLY.

This package restates, in FP64 NumPy/SciPy, the algorithm of the reference
Fortran solver (MetamaterialFSI/channel3D_parallel, ``src/*.f90``) for the hot
path ``compute_time_step_RK3`` and everything it calls.  Every function cites
the reference file:line it follows.

Status: **parity unpinned**.  The reference ships no tests, golden vectors or
fixtures for this path, and it cannot be compiled in this container (no
Fortran compiler, MPI, FFTW or system LAPACK).  The restatement is pinned
instead by known-answer tests derived from the mathematics (single Fourier
modes through the Poisson solve, Poiseuille balance, delta-function moment
identities, E/R adjointness, ...) under ``tests/``.

``cpu_rk3.cpp`` (with its ctypes wrapper ``cpu_rk3.py``) restates the same
FP64 RK3 step in C++/OpenMP; it is the timed CPU baseline of ``bench.py`` and
is itself checked against the NumPy restatement.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker or as the timed CPU
baseline.  The product path (``channel3d_parallel_b200``) never imports it.
"""
