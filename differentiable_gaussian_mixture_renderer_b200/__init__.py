"""B200-native differentiable Gaussian-mixture rendering (splat + vol_marcher)."""
