// fy_deconv_ct_a.cu -- compile-time-plan deconvolution passes for axis lengths 512, 96, 1024.
#include "fy_deconv.cuh"

cudaError_t fy_deconv_pass_ct_a(int pass, int n, const DeconvLaunch& d, cudaStream_t st) {
    switch (n) {
        FY_DECONV_CT_CASE(512) FY_DECONV_CT_CASE(96) FY_DECONV_CT_CASE(1024)
        default: return cudaErrorNotSupported;
    }
}

int fy_deconv_ct_a_timeouts() { return dc_timeouts(); }
