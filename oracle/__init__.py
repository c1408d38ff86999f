"""The oracle: CPU restatements to check the CUDA timestep against.  TEST
INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only to check results against (or as
the timed CPU baseline), never as the thing measured or shipped.

* ``Oracle``    — the project's own C restatement of the reference timestep
                  (``acg_oracle.c``), built to ``oracle/_build/libacg_oracle.so``.
* ``Reference`` — the reference's own MDcode sources compiled in place with a
                  single-rank MPI shim and a GSL shim (``Makefile``), built to
                  ``oracle/_ref/libref_md_n<N>.so`` (one library per N because
                  the reference fixes N at compile time).  Present only where
                  the reference sources were available when the repo was built.
* ``observables`` — numpy restatement of the reference's trajectory analysis
                  (overlap Q(t), chi4, MSD) used to check the in-place
                  accumulators.
"""
from .bindings import Oracle, Reference, build_oracle, oracle_lib_path, reference_available, ref_lib_path  # noqa: F401
