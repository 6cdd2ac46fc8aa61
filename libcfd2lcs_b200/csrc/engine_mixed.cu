// The mixed-precision form of the double library's engine: velocity levels, their spline
// coefficients and the stage blends in FP32, everything else in the interface type (see
// class Engine in engine_impl.cuh).  Compiled apart from engine.cu so that the two template
// instantiations build in parallel; the single library needs no separate form (its interface
// type is already FP32).
#include "engine_impl.cuh"

namespace cfd2lcs {

#ifndef CFD2LCS_SP
std::unique_ptr<EngineBase> make_engine_mixed(const Options *opt) { return std::unique_ptr<EngineBase>(new Engine<float>(opt)); }
#endif

}  // namespace cfd2lcs
