"""CPU oracle for the multiple-double power-series path (test infrastructure).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this
package, and only as the checker.  The product never calls it.
"""
