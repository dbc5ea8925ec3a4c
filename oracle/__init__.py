"""CPU oracle of the DSMC hot path (test infrastructure only; see oracle/oracle.py)."""
