"""The oracle: CPU restatement of the reference's Jacobi-PCG path, plus the reference's own
sources built as oracle/_ref/libxplus_ref.so.  TEST INFRASTRUCTURE ONLY -- imported by
tests/, __graft_entry__.smoke() and bench.py's CPU baseline; never by the product."""
