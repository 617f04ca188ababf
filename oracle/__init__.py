"""CPU oracle for the RAISHIN GRMHD update (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, as the checker.  The product (raishinsource_b200) never imports it.
Parity status: unpinned (the reference ships no golden data and cannot be
compiled here); see oracle/oracle.hpp.
"""
from .pyoracle import Oracle, build, pow_eval, set_pow_mode  # noqa: F401
