"""B200-native Redi neutral-diffusion step (ocean_redi) behind the reference's entry points."""
