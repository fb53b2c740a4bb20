"""CPU checkers for the ECSG CUDA path.  TEST INFRASTRUCTURE ONLY.

* ``oracle.oracle``  -- ctypes front end of the project's C restatement
  (ecsg_oracle.c) plus numpy restatements of the reference's set-up steps and
  of main.cpp's time loop.
* ``oracle.ref``     -- ctypes front end of the reference itself, compiled from
  its own sources into oracle/_ref/ (see oracle/Makefile).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  The product package ecsg_b200 never does.
"""
