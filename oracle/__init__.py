"""CPU oracle for the integrating-factor RK3 pseudo-spectral step.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path imports this package:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, and only as the checker or
as the timed CPU reference arm.

Contents
--------
``spectral_oracle``
    FP64 NumPy restatement of the reference solver ``reference/spectral2d.py``
    (the vorticity-streamfunction RK3 step, diagnostics and the band-limited
    random field).  Pinned against the reference's own golden vectors
    (``tests/fixtures.json`` of the reference, re-exported under
    ``tests/golden/``) and against outputs of ``reference/spectral2d.py`` run
    in the development container (``tests/golden/make_golden.py``).
``fft_oracle``
    Restatement of ``reference/fft_ref.py``: radix schedule, digit reversal
    over the reversed radix list and the in-place DIT line model.  Pinned
    against the digit-reversal tables and line transforms produced by
    ``reference/fft_ref.py``.
``wgsl_oracle``
    NumPy restatement of the parts of the step that exist only as WGSL / JS in
    the reference (stochastic forcing, pointer forcing, CFL reduction, dye
    advection, spectral seeding, dye painting, fixed-point diagnostics).  The
    reference has no test, fixture or runnable CPU code for these: their
    parity is UNPINNED (checked only against this restatement).
"""
