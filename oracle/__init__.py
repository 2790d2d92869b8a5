"""TEST INFRASTRUCTURE ONLY: the CPU oracle for the Gibbs-sweep hot path (see oracle.py)."""
