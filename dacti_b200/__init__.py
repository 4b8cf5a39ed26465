"""B200-native octree finite-volume step (Euler / Navier-Stokes / five-equation multiphase)."""
