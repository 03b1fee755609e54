// fnec_mixed.cu -- mixed-precision path (not built yet).
#include "fnec_mixed.h"

namespace fnec {

bool mixed_available() { return false; }
cudaError_t alloc_mixed(MixedWork &w, const std::vector<UnitDesc> &, int) {
    w.bytes = 0;
    return cudaSuccess;
}
void free_mixed(MixedWork &w) {
    if (w.base) cudaFree(w.base);
    w.base = nullptr;
}
uint64_t run_mixed(MixedWork &, const UnitDesc *, int, const std::vector<UnitDesc> &, const AntDesc *,
                   const DevSeg *, const int4 *, int, const int4 *, int, const int32_t *,
                   const DevConstraint *, const int32_t *, cx *, const cx *, const double *, cx *, cx *,
                   int32_t *, int32_t *, int, bool, MixedMarks, cudaStream_t) {
    return 0;
}

}  // namespace fnec
