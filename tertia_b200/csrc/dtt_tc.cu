// dtt_tc.cu — split-precision tensor-core transforms (see dtt_tc.h).
#include "dtt_tc.h"
#include "qs_common.cuh"

namespace qs {

TcTransformer* TcTransformer::create(int mode, int ny, int nz, cudaStream_t st,
                                     std::string& why) {
    (void)mode; (void)ny; (void)nz; (void)st;
    why = "split-precision tensor-core transforms are not built yet";
    return nullptr;
}

}  // namespace qs
