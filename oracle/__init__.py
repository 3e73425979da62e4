"""CPU oracles of the kernel-integral path -- test infrastructure only (see oracle/oracle.py)."""
