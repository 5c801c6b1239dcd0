"""B200-native drop-in for the ESyS-Particle per-timestep DEM hot path (``esys.lsm``)."""
