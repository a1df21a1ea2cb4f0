"""GraGLeS2D's per-timestep level-set grain-growth update on one B200."""
