"""Test infrastructure: the CPU oracle for the ADMM solve loop.

* ``liboracle.so`` -- the C restatement of the reference algorithm
  (``wrapd_oracle.c``), built by ``make -C oracle oracle``.
* ``_ref/quasi_ref`` and ``_ref/libref_elem.so`` -- the reference itself, built
  from the reference sources by ``make -C oracle ref`` (only where the sources
  are present; the built files travel with the repository snapshot).

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline use
this package, as the checker.  The product never imports it.
"""
from .pyoracle import (Oracle, OracleProblem, load_oracle, load_ref_elem, ref_available,
                       run_quasi_ref, QUASI_REF, ORACLE_DIR)

__all__ = ["Oracle", "OracleProblem", "load_oracle", "load_ref_elem", "ref_available",
           "run_quasi_ref", "QUASI_REF", "ORACLE_DIR"]
