"""Oracle for the H-matrix matvec -- TEST INFRASTRUCTURE ONLY.

Two checkers live here:

* ``RefHmat``: the unmodified reference library (``_ref/libbigwham_ref.so``,
  compiled from the reference sources by ``oracle/Makefile``) driven through
  ``ref_capi.cc``.  It builds H-matrices with the reference's own code and runs
  the reference's own OpenMP CPU matvec (``BigWhamIO::MatVec``,
  src/io/bigwham_io.cc:927-933).
* ``oracle_*``: a plain-C restatement of ``Hmat::matvec`` /
  ``matvecOriginal`` (src/hmat/hmatrix/hmat.cc:472-635) over flat arrays
  (``_lib/libhmat_oracle.so``), pinned against the reference by the golden
  vectors in tests/golden.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product never calls it.
"""
from .pyoracle import (  # noqa: F401
    HmatArrays,
    RefGaussian,
    RefHmat,
    oracle_available,
    oracle_diagonal,
    oracle_entries,
    oracle_matmat,
    oracle_matvec,
    oracle_matvec_perm,
    oracle_rmatvec,
    oracle_rmatvec_perm,
    ref_available,
)
