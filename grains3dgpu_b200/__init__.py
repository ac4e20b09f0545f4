"""B200-native DEM time step behind Grains3D's ComponentManager interface."""
