"""Checkers for the mach_b200 CUDA path (test infrastructure only).

* das_fp64.py   -- FP64 NumPy restatement of mach's DAS arithmetic
* das_oracle.c  -- the same in C with OpenMP (also the timed CPU baseline)
* ref_shim/     -- builds mach's own CUDA kernel from its unmodified source
* machref.py    -- ctypes front end for that reference build

Only tests/, __graft_entry__.smoke() and bench.py's baseline legs use this package.
"""
