// tune.cu -- autotuner: per problem fingerprint, the measured-best design-
// space point.  The reference has no selector (the caller passes alg,
// spmvspmm.h:57-58); DASPMM_ALG_AUTO uses this cache, falling back to a rule
// of thumb before anything has been measured.
#include "internal.h"

namespace daspmm {

daspmm_status tuned_config(int layout, int nr, int nc, int nnz, int nv, daspmm_config *out)
{
    (void)nc;
    daspmm_config c{};
    // Rule of thumb: nonzero-balanced CSR for wide dense operands (rows of B
    // are >= 128 bytes, so one group per chunk streams whole B rows), the
    // row-balanced scalar kernel otherwise.
    c.alg = (layout == DASPMM_ROW_MAJOR && nv >= 32) ? DASPMM_ALG_CSR_BALANCED
                                                      : DASPMM_ALG_CSR_SCALAR;
    Resolved r;
    daspmm_status s = resolve(&c, layout, nr, nnz, nv, nullptr, nullptr, &r);
    if (s != DASPMM_OK) return s;
    *out = to_config(r);
    return DASPMM_OK;
}

}  // namespace daspmm
