/*
 * Discrete adjoint of the RK2 MHD step: host checks of the pointwise
 * vector-Jacobian products and (below) the reverse-pass kernels.
 */
#include <cuda_runtime.h>

#include "../../include/fornax_b200.h"
#include "fx_adjoint.cuh"

namespace {

void face_out_pack(const FxFaceOut &o, double *out)
{
    for (int v = 0; v < 9; ++v) {
        out[v] = o.F[v];
    }
    out[9] = o.v[0];
    out[10] = o.v[1];
    out[11] = o.v[2];
    out[12] = o.bv1;
    out[13] = o.bv2;
}

} // namespace

extern "C" int fx_face_eval_host(const double *w4, double bn, double gamma, double *out)
{
    if (!w4 || !out || !(gamma > 1.0)) {
        return FX_EINVAL;
    }
    FxFaceOut o;
    fxa_face_eval(w4, gamma, bn, o);
    face_out_pack(o, out);
    return FX_SUCCESS;
}

extern "C" int fx_face_vjp_host(const double *w4, double bn, double gamma, const double *out_bar,
    double *w4_bar, double *bn_bar)
{
    if (!w4 || !out_bar || !w4_bar || !bn_bar || !(gamma > 1.0)) {
        return FX_EINVAL;
    }
    for (int n = 0; n < 36; ++n) {
        w4_bar[n] = 0.0;
    }
    double bnb = 0.0;
    fxa_face_vjp(w4, gamma, bn, out_bar, w4_bar, bnb);
    *bn_bar = bnb;
    return FX_SUCCESS;
}
