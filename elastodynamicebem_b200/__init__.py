"""B200-native energetic space-time Galerkin BEM for 3D elastodynamics."""
