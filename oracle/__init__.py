"""CPU oracle for the ExaGeoStatCPP maximum-likelihood path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
package; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg use it, and there only as the checker.
"""
