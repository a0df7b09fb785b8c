"""CPU oracle of the SBP path: test infrastructure only (see sbp_oracle.cpp)."""
