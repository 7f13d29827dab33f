"""FP64 CPU oracle for the imaging-and-gradient hot path.

TEST INFRASTRUCTURE ONLY. This package restates, in float64 NumPy/SciPy, the
reference C++ code of wyhcoder/C-version-Lithography for the SOCS imaging,
the pattern-error loss and its adjoint, the CTM theta chain and the
WENO5-Godunov level-set update. Every function cites the reference file:line
it follows. Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it,
and only as the checker or the timed CPU restatement; the product path in
``c-version-lithography_b200`` never calls it.

The reference cannot be compiled here (Eigen, FFTW, OpenCV-C++, yaml-cpp and
LBFGS++ are absent), so this restatement is pinned against the reference's
own known-answer tests instead (``tests/test_oracle_pins.py``): the Godunov
planar / extremum / circle-symmetry cases of
``tests/test_level_set_godunov.cpp``, the finite-difference gradient checks
of ``tests/test_ctm_optimizer.cpp:61-96`` on real optics, the compact-vs-dense
SOCS equality of ``tests/test_full_chip_imaging_compare.cpp:83-103`` and the
partition geometry of ``tests/test_micro_gradient_exchange.cpp``. The L-BFGS
trajectory (LBFGS++ v0.4.0) is not pinned; only its stopping behaviour is.
"""
