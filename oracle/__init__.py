"""CPU oracle for the closed-shell coupled-cluster path.

TEST INFRASTRUCTURE ONLY. This package is a numpy restatement of ElemCo.jl's
closed-shell CCSD/DCSD residual, amplitude updates, DIIS, (T), Lambda-(T) and
Lambda equations. It is the checker for the CUDA library: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
The product path (``ecgpu`` + ``libecgpu.so``) never calls into it.

Parity pin: the oracle reproduces the reference's pinned energies
(ElemCo.jl test/h2o.jl:6-10, test/h2o_st1.jl:6-9) from the reference's own
FCIDUMP fixtures, see ``tests/test_oracle_golden.py``.
"""
from .ccref import *  # noqa: F401,F403
