"""CPU oracle for the retarded BEM solve per wavelength -- TEST INFRASTRUCTURE.

This package restates, in numpy/scipy complex128, the reference algorithm of
the path that ``mnpbem_b200`` runs on the GPU (MNPBEM, Python port v1.6.2):

* refinement matrix, polar / 28-point refinement integrals, closed-surface
  correction                     -> ``oracle.green``  (a1-a5)
* Green matrices G1, G2, H1, H2  -> ``oracle.green``  (a6)
* BEMRet init / excitation / solve, full 8N operator -> ``oracle.bem`` (a7-a10)
* plane-wave potentials, far field, extinction, scattering -> ``oracle.farfield``
* transposed solve and reverse-mode geometry derivatives (no reference
  counterpart; checked by adjoint identities)        -> ``oracle.adjoint``

Every function cites the reference file:line it follows.  The oracle is
pinned against golden vectors produced by the reference itself
(``tests/golden/make_golden.py``) and against MNPBEM17's MATLAB results
committed in the reference (validation/03_bemret/sphere/data/bemret_matlab.csv).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package, and only as the checker / the timed CPU baseline.
The product path (``mnpbem_b200``) never imports it.
"""
