"""Oracle for the RelaxMap hot path: TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs may import this package. The product (relaxmap_b200) never does.
"""
