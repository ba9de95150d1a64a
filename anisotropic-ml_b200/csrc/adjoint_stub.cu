#include "common.cuh"
extern "C" amlp_status amlp_forces_adjoint(const float *, const float *, float, const int *, const long long *,
                                           long long, const amlp_nep *, const amlp_mlp *, float *, float *,
                                           double *, void *) {
    return AMLP_ERR_UNSUPPORTED;
}
