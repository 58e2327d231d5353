"""Test infrastructure only: the CPU oracle for the fermion-solve hot path.

``load_oracle()`` returns the C restatement (oracle.c) and ``load_reference()``
the reference's own kernels compiled from its sources (Makefile target
``ref``).  Only tests/, the smoke check and the bench's CPU-baseline leg use
them, always as the checker, never as the thing measured or shipped.
"""
from .loader import (  # noqa: F401
    OracleGeom, load_oracle, load_reference, reference_available, build_oracle, build_reference,
)
