"""CPU oracle of the PCOM time step -- test infrastructure only (see pcom_oracle.cpp)."""
