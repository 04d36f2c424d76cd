"""CPU oracle for the Goldilocks commit path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg import
this package; the zeknox_b200 library never does.
"""
