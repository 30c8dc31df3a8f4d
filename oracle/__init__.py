"""CPU oracle for the accusim short-range force-and-step path.

TEST INFRASTRUCTURE ONLY. This package is the checker: it is imported by `tests/`, by
`__graft_entry__.smoke()` and by the CPU-baseline / `--impl reference` legs of `bench.py`, and by
nothing else. The product path (`devinproj_b200`) never imports it and has no CPU fallback.

`accusim_port` restates, in NumPy FP64, the reference algorithm of accusim (erezbz/DevinProj,
package `accusim`): cell-list pairs, the Verlet skin list, Lennard-Jones with Lorentz-Berthelot
mixing and a shifted cutoff, damped-shifted-force Coulomb, Ewald (label oracle), VelocityVerlet,
the conserved-quantity reductions and the accuracy-report drift metrics. Every function cites the
reference file:line it follows.

Parity pin: `tests/test_oracle_golden.py` checks this port against golden vectors generated by the
reference itself (`tests/golden/make_golden.py`, run where the reference is importable) and against
the reference's own known answers (Madelung constant, LJ minimum at 2^(1/6) sigma).
"""
