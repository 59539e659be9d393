// eloc_kb2.cu -- instantiations of the FP32 evaluation kernel (eloc.cuh) for
// groups of 2 hidden units.
#include "eloc.cuh"

namespace rbmnqs {
namespace eloc {

const void* pick_kb2(int ng, bool sym, int nfm) {
    switch (ng) {
        case 1: return pick3<2, 1>(sym, nfm);
        case 2: return pick3<2, 2>(sym, nfm);
        case 4: return pick3<2, 4>(sym, nfm);
        case 8: return pick3<2, 8>(sym, nfm);
    }
    return nullptr;
}

}  // namespace eloc
}  // namespace rbmnqs
