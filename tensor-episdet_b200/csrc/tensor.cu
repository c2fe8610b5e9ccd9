// tensor.cu -- tcgen05 (5th-generation tensor core) counting engine.
#include "search_internal.h"
#include "host_util.h"

namespace episdet {

episdet_status run_tensor(Workspace* w, DevData& D, const ScoreTables& T, const episdet_options& o, int fb, int fe,
                          Slots* S, uint64_t* launches, bool progress) {
    (void)w; (void)D; (void)T; (void)o; (void)fb; (void)fe; (void)S; (void)launches; (void)progress;
    return set_error(EPISDET_ERR_UNSUPPORTED, "tensor engine not built");
}

}  // namespace episdet
