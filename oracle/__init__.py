"""CPU checkers for the AdaptFlood time step (test infrastructure only)."""
