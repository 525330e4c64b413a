"""CPU parity oracle for hsolver's SIMPLE-CHT outer step (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker or the timed CPU baseline; the product in
hsolver_b200/ never imports it.
"""
