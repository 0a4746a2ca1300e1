"""CPU oracle for the DSEM hot path (test infrastructure, the checker).

Only tests, the smoke check and the CPU-baseline leg of bench.py import this
package.  The product (dsem_b200) never imports, loads or calls it.
"""
