"""B200-native CUDA backend for the inundation shallow-water step."""
