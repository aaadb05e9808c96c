"""CPU oracle (test infrastructure): see oracle/oracle.py and oracle/cnm_oracle.cpp."""
