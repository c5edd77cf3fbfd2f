// TEST INFRASTRUCTURE (oracle).  Stand-in for Random123's uniform.hpp: only u01<float>.
#ifndef FR_ORACLE_SHIM_UNIFORM_HPP
#define FR_ORACLE_SHIM_UNIFORM_HPP
#include <cstdint>
#include "../restated_math.hpp"
namespace r123 {
template <typename Ftype, typename Itype> inline Ftype u01(Itype in)
{
    return frm::u01(uint32_t(in));
}
}  // namespace r123
#endif
