"""ORACLE / TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.

`oracle.oracle` is the plain-C restatement of the reference stepper (twave_oracle.c);
`oracle.refrun` drives the reference's own CPU solvers compiled into oracle/_ref.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference legs use them.
"""
