"""B200-native 3DGS preprocess/bin/sort/raster/backward hot path (see include/gs3d_cuda.h)."""
