"""CPU oracles of the walk-on-spheres path (test infrastructure only): the
plain-C restatement (wos_oracle.c) and the reference compiled from its own
sources (oracle/_ref).  See oracle/oracle.py."""
