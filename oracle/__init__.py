"""CPU oracle for the nricp wrapping path -- test infrastructure only.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker; the product (nricp_b200) never imports it.
"""
