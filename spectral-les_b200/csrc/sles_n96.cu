// Kernel instantiations for N = 96 (float32/float64, 2D and 3D).
#include "sles_engine.cuh"
SLES_DEFINE_ENGINES(96)
