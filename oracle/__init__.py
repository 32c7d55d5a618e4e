"""The oracle: CPU reference implementations of the time step (test infrastructure only)."""
