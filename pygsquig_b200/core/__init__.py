"""Grid, solver and time stepping of the gSQG hot path."""
