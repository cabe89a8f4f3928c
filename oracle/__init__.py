"""CPU oracle for the dynamical core (TEST INFRASTRUCTURE ONLY; see model.py, oracle.c, build_ref.py)."""
