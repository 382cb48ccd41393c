"""CPU oracle for lbman3d's per-timestep path (test infrastructure only)."""
