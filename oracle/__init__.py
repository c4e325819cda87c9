"""CPU oracle for the CAMP per-cell chemistry solve — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package, and only as the checker.  The product (camp_b200) never
imports it and has no CPU fallback.
"""
