"""Oracle package — TEST INFRASTRUCTURE ONLY.

CPU restatements of the reference's Trotter sampler path used as the checker for
the CUDA engine. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may
import this package; the product never does.
"""
