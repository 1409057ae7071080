"""Scalar CPU oracle of the Amethyst operator layer -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py may import this
package, and only as the checker.  The product (amethyst_b200, libamethyst_b200.so) never
imports, links or executes anything here.
"""
