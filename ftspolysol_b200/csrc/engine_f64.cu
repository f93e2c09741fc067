// Complex128 instantiation of the engine.
#include "engine.cuh"

namespace ftsp {
EngineBase* make_engine_f64(const HostCfg& c) { return new Engine<double>(c); }
}  // namespace ftsp
