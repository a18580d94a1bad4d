"""CPU oracle of the implicit stepping path -- TEST INFRASTRUCTURE, NOT THE PRODUCT.

A numpy/scipy restatement of the reference's residual (core/residual.py with physics/,
boundaries/, properties/), coloured finite-difference Jacobian (core/jacobian.py,
numerics/sparsity.py) and 2-stage implicit Runge-Kutta Newton-Krylov integrator
(core/solver.py).  Every function cites the reference file:line it follows.

Pinned against golden vectors generated by importing the reference itself
(tests/golden/make_golden.py) and against the reference's own known-answer tests
(isotherm values, conservation, T<->e round trip, colouring validity).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may
import this package; the GPU product path never does.
"""
