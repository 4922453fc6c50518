"""CPU parity oracle for the MOM6 split RK2 step (test infrastructure only).

Only tests/, the smoke check and bench.py's cpu_baseline leg may import this
package.  It wraps oracle/liboracle.so, a C restatement of the reference's
serial Fortran path (see oracle/mom6_oracle.h).
"""
