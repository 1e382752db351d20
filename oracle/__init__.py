"""CPU oracle for the LATEC plain-codec hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU, the algorithm of the reference LATEC code for
the path the CUDA library implements: the dyadic stage schedule, the
cubic/linear interpolation predictor, the error-bounded quantizer, the
Laplace-mixture rANS model tables, the per-point rANS coder (``point.py``)
and the LATEC001 container. Each function
cites the reference file and line it follows (paths relative to the reference
project root).

Parity pinning: the NumPy parts are checked against golden vectors generated by
running the reference package itself (``tests/golden/make_golden.py``) --
schedules, per-stage codes/outliers/reconstructions, predictions, quantizer
outputs and rANS tables. The byte-level rANS coder (``ans.c``) restates the
published stack-ANS algorithm of the ``constriction`` 0.4 crate, which the
reference calls but which is absent here; no reference test pins coder bytes,
so the compatibility byte stream is *parity unpinned* (round trips and
model-bit tracking are checked instead).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker / the timed CPU baseline.
The product (``latec_b200``) never imports it and has no CPU fallback.
"""
