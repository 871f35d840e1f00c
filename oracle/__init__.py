"""CPU oracle for the dsDecompX particle-bookkeeping hot path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py`` (its ``cpu_baseline`` leg and ``--impl reference`` arm), never
by the ``dsdecompx_b200`` package.

Two backends share one Python interface (:class:`Grid`):

* ``"port"`` -- ``dsx_oracle.c``, a plain-C restatement of the reference's
  Host-mode algorithm for P virtual subdomains in one thread;
* ``"ref"`` / ``"ref_debug"`` -- the reference's own Host-path sources,
  compiled unmodified against the in-process thread-per-rank MPI stand-in
  (``mpi_shim/``), one thread per rank.  ``ref_debug`` keeps the reference's
  debug invariants (id uniqueness/conservation, owner-domain check) on.

The port is pinned against ``ref`` by the CPU test suite and by the golden
fixtures in ``tests/golden``.
"""
from .oracle import (ARRAYS, FIELD_DTYPES, OPS, POLICIES, Grid, available,
                     library_path)

__all__ = ["ARRAYS", "FIELD_DTYPES", "OPS", "POLICIES", "Grid", "available",
           "library_path"]
