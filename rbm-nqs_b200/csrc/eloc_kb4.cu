// eloc_kb4.cu -- instantiations of the FP32 evaluation kernel (eloc.cuh) for
// groups of 4 hidden units.
#include "eloc.cuh"

namespace rbmnqs {
namespace eloc {

const void* pick_kb4(int ng, bool sym, int nfm) {
    switch (ng) {
        case 1: return pick3<4, 1>(sym, nfm);
        case 2: return pick3<4, 2>(sym, nfm);
        case 4: return pick3<4, 4>(sym, nfm);
    }
    return nullptr;
}

}  // namespace eloc
}  // namespace rbmnqs
