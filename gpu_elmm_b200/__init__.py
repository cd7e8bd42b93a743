"""B200-native per-timestep flow solve of the ELMM LES model."""
