// eloc_kb1.cu -- instantiations of the FP32 evaluation kernel (eloc.cuh) for
// groups of 1 hidden unit.
#include "eloc.cuh"

namespace rbmnqs {
namespace eloc {

const void* pick_kb1(int ng, bool sym, int nfm) {
    switch (ng) {
        case 2: return pick3<1, 2>(sym, nfm);
        case 4: return pick3<1, 4>(sym, nfm);
        case 8: return pick3<1, 8>(sym, nfm);
        case 16: return pick3<1, 16>(sym, nfm);
    }
    return nullptr;
}

}  // namespace eloc
}  // namespace rbmnqs
