"""Oracle (test infrastructure only; never imported by the product).

* ``oracle/Makefile`` compiles the unmodified nuTRLan reference from its own
  sources into ``oracle/_ref/libnutrlan_ref.so`` (serial backend, OpenBLAS).
* ``oracle.ref`` drives that library through ctypes with numpy operators.
* ``oracle.kernels_np`` restates the hot-path vector operations (CGS
  projection/update, Ritz recombination, CSR product, the alpha dot) in
  numpy FP64, each citing the reference code it follows.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may use this package, and only as the checker or the CPU
baseline.
"""
