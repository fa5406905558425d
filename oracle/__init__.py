"""CPU checkers for the Louvain path (test infrastructure only).

``oracle.c_oracle`` wraps the C restatement (liblvoracle.so) and
``oracle.reference`` wraps Grappolo's own functions compiled from its sources
(_ref/libgrappolo_ref.so).  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py use them, and only as checkers.
"""
from .lvoracle import COracle, Reference, PhaseRecord, build  # noqa: F401
