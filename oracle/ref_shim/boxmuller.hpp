// TEST INFRASTRUCTURE (oracle).  Stand-in for Random123's boxmuller.hpp.  The reference calls
// boxmuller only from RayGen::uniformSampleReflection (fresnel/common/RayGen.h:71-100), which no
// tracer calls; the stub exists so that the header compiles.
#ifndef FR_ORACLE_SHIM_BOXMULLER_HPP
#define FR_ORACLE_SHIM_BOXMULLER_HPP
#include <cstdint>
namespace r123 {
struct float2 {
    float x, y;
};
inline float2 boxmuller(uint32_t, uint32_t) { return float2{0.0f, 0.0f}; }
}  // namespace r123
#endif
