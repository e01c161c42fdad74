// Kernel instantiations for N = 512 (float32/float64, 2D and 3D).
#include "sles_engine.cuh"
SLES_DEFINE_ENGINES(512)
