// FP32-mixed engine: fields, stencils, HSMAC sweeps and the fluid velocity
// seen by particles in FP32; the HSMAC residual and convergence test, the
// energy and dissipation reductions behind the forcing, the time step and the
// particle state stay FP64.  No reference counterpart (the reference computes
// in `const FP = Float64`, src/LCS.jl:20); FMA contraction is allowed here.
#include "lcs_engine.cuh"

namespace lcs {
EngineBase* make_engine_f32(const lcs_config& c, std::string* err, int* rc) {
  Engine<float>* e = new Engine<float>();
  *rc = e->init(c);
  if (*rc != LCS_OK) {
    *err = e->err;
    delete e;
    return nullptr;
  }
  return e;
}
int64_t footprint_f32(const lcs_config& c) { return (int64_t)make_plan<float>(c).bytes; }
}  // namespace lcs
