// TEST INFRASTRUCTURE (oracle).  Stand-in for Random123's philox.h, which the reference
// includes from its extern/random123 submodule (absent from the reference tree).  Only the
// names the reference's common/*.h headers use are provided; the generator is the published
// Philox4x32-10 algorithm, implemented once in restated_math.hpp.
#ifndef FR_ORACLE_SHIM_PHILOX_H
#define FR_ORACLE_SHIM_PHILOX_H
#include <cstdint>
#include "../../restated_math.hpp"

namespace r123 {
struct Array2x32 {
    uint32_t v[2];
};
struct Array4x32 {
    uint32_t v[4];
};
struct Philox4x32 {
    typedef Array4x32 ctr_type;
    typedef Array2x32 key_type;
    typedef Array2x32 ukey_type;
    ctr_type operator()(ctr_type c, key_type k) const
    {
        frm::Ctr4 in{{c.v[0], c.v[1], c.v[2], c.v[3]}};
        frm::Ctr4 out = frm::philox4x32_10(in, k.v[0], k.v[1]);
        ctr_type r{{out.v[0], out.v[1], out.v[2], out.v[3]}};
        return r;
    }
};
}  // namespace r123
#endif
