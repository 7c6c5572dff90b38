"""B200-native 3D Gaussian Splatting training and render path (msplat backend)."""
