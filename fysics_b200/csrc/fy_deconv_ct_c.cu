// fy_deconv_ct_c.cu -- compile-time-plan deconvolution passes for axis lengths 128, 192, 768.
#include "fy_deconv.cuh"

cudaError_t fy_deconv_pass_ct_c(int pass, int n, const DeconvLaunch& d, cudaStream_t st) {
    switch (n) {
        FY_DECONV_CT_CASE(128) FY_DECONV_CT_CASE(192) FY_DECONV_CT_CASE(768)
        default: return cudaErrorNotSupported;
    }
}

int fy_deconv_ct_c_timeouts() { return dc_timeouts(); }
