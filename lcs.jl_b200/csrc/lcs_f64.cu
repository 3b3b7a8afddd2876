// FP64 engine: the reference's arithmetic.  Built with --fmad=false so every
// element-wise result equals the CPU restatement bit for bit.
#include "lcs_engine.cuh"

namespace lcs {
EngineBase* make_engine_f64(const lcs_config& c, std::string* err, int* rc) {
  Engine<double>* e = new Engine<double>();
  *rc = e->init(c);
  if (*rc != LCS_OK) {
    *err = e->err;
    delete e;
    return nullptr;
  }
  return e;
}
int64_t footprint_f64(const lcs_config& c) { return (int64_t)make_plan<double>(c).bytes; }
}  // namespace lcs
