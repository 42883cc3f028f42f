// TEST INFRASTRUCTURE ONLY (the oracle). Links the seeded synthetic scene
// generators (the package's csrc/vgi_scenes.cpp, compiled a second time into
// liboracle.so by oracle/Makefile) to the oracle's own hashing, so that
// bench.py's CPU arm and the tests can make the benchmark scenes without
// loading the product library. The generators are input synthesis, not part
// of the traced path: the terrain, cave and face lists they write are the same
// bytes in both libraries.
#include "oracle.h"
#include "vgi_runtime.h"

namespace vgi {

uint32_t host_pcg(uint32_t v) { return orc::pcg(v); }

size_t RegionKeyHash::operator()(const RegionKey& k) const { return orc::hash_voxel(k.x, k.y, k.z); }

}  // namespace vgi
