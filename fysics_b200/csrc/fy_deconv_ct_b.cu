// fy_deconv_ct_b.cu -- compile-time-plan deconvolution passes for axis lengths 256, 384, 64.
#include "fy_deconv.cuh"

cudaError_t fy_deconv_pass_ct_b(int pass, int n, const DeconvLaunch& d, cudaStream_t st) {
    switch (n) {
        FY_DECONV_CT_CASE(256) FY_DECONV_CT_CASE(384) FY_DECONV_CT_CASE(64)
        default: return cudaErrorNotSupported;
    }
}

int fy_deconv_ct_b_timeouts() { return dc_timeouts(); }
