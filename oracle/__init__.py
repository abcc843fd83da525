"""CPU oracle for the density-fitting contraction path (TEST INFRASTRUCTURE).

This package is the checker, never the product. It restates, in NumPy/SciPy
FP64, the reference algorithms that ``libferric_cuda`` replaces:

* ``oracle.rimp2``   -- closed-shell RI-MP2 spin components, the 3-index
  adjoint Gamma = dE/dB and dE/d(eps)
  (ferric-mp2/src/rimp2.rs, oo_rimp2.rs, zvector.rs);
* ``oracle.dfjk``    -- DF-J (packed two-pass with metric solve) and DF-K
  (occupied half-transform path and density path)
  (ferric-scf/src/df_j.rs, df_k.rs);
* ``oracle.synthetic`` -- seeded generators of the synthetic workloads;
* ``oracle.basis`` / ``oracle.integrals`` / ``oracle.scf`` -- a small
  Gaussian-integral engine and RHF used only to pin this oracle to the
  reference's PySCF golden energies for water.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg and
``--impl reference`` arm of ``bench.py`` may import it.  The product package
``ferric_b200`` never imports it and has no CPU fallback.
"""
