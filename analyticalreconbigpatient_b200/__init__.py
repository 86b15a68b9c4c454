"""B200-native helical cone-beam FBP chain (rebin -> preweight/ramp filter -> 3D-weighted backprojection)."""
