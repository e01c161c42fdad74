// Kernel instantiations for N = 1024 (2D only: a 1024^3 field set exceeds the
// workspace budget this library targets).
#include "sles_engine.cuh"
namespace sles {
Engine* make_engine_1024(int dtype, int dim) {
  if (dim != 2) return nullptr;
  if (dtype == SLES_F32) return new EngineImpl<float, 1024, 2>();
  if (dtype == SLES_F64) return new EngineImpl<double, 1024, 2>();
  return nullptr;
}
}  // namespace sles
