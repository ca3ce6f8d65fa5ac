"""Test infrastructure: the CPU oracle of the MPulse hot path (see mpulse_oracle.c)."""
