// Complex64 instantiation of the engine.
#include "engine.cuh"

namespace ftsp {
EngineBase* make_engine_f32(const HostCfg& c) { return new Engine<float>(c); }
}  // namespace ftsp
