// fy_deconv.cu -- the five deconvolution passes (fy_deconv.cuh) on the runtime plan, the
// dispatch to the compile-time instantiations, and the Y pass shared with phase correlation.
#include "fy_deconv.cuh"

namespace {
// axis length of each pass: 1/5 x, 2/4 y, 3 z
int pass_len(int pass, const SpecGeom& g) { return pass == 3 ? g.pz : (pass == 2 || pass == 4) ? g.py : g.px; }
const char* const kPassName[6] = {"", "deconv.x_fwd", "deconv.y_fwd", "deconv.z_weight", "deconv.y_inv", "deconv.x_inv"};
}  // namespace

size_t fy_deconv_spec_elems(const SpecGeom& g) { return (size_t)g.nz * g.py * g.hxp; }

cudaError_t fy_launch_deconv(const DeconvLaunch& d, cudaStream_t st) {
    for (int pass = 1; pass <= 5; ++pass) {
        const int n = pass_len(pass, d.g);
        cudaError_t e = fy_deconv_pass_ct_a(pass, n, d, st);
        if (e == cudaErrorNotSupported) e = fy_deconv_pass_ct_b(pass, n, d, st);
        if (e == cudaErrorNotSupported) e = fy_deconv_pass_ct_c(pass, n, d, st);
        if (e == cudaErrorNotSupported) e = fy_deconv_pass<0>(pass, d, st);
        if (e != cudaSuccess) return e;
        fy_prof_mark(st, kPassName[pass]);
    }
    return cudaSuccess;
}

// Y pass over `nplanes` stored planes of a half spectrum (shared with phase correlation):
// sign -1 forward (rows >= ny gathered by reflection or zero), +1 inverse keeping rows
// < keep_rows.
cudaError_t fy_launch_spec_y(float2* spec, const SpecGeom& g, const FftPlan& ply, const float2* twy, int nplanes,
                             int sign, int keep_rows, cudaStream_t st) {
    const TileShape t = fy_tile_shape(g.py);
    const size_t smem = (size_t)g.py * t.W * sizeof(float2) + (size_t)g.py * sizeof(float2);
    dim3 grid(ceil_div_i(g.hx, t.W), nplanes);
    return fy_with_e(t.E, [&](auto ec) -> cudaError_t {
        constexpr int E = decltype(ec)::value;
        if (sign < 0) {
            auto k = k_y_fwd<0, E>;
            cudaError_t e2 = fy_smem_optin(k, smem);
            if (e2 != cudaSuccess) return e2;
            k<<<grid, t.NT, smem, st>>>(spec, g, ply, twy, t.wlog);
        } else {
            auto k = k_y_inv<0, E>;
            cudaError_t e2 = fy_smem_optin(k, smem);
            if (e2 != cudaSuccess) return e2;
            k<<<grid, t.NT, smem, st>>>(spec, g, ply, twy, keep_rows, t.wlog);
        }
        return cudaGetLastError();
    });
}

// Expired bulk waits of the deconvolution's first pass in every unit that instantiates it.
int fy_deconv_wait_timeouts() {
    const int v[4] = {dc_timeouts(), fy_deconv_ct_a_timeouts(), fy_deconv_ct_b_timeouts(), fy_deconv_ct_c_timeouts()};
    int t = 0;
    for (int x : v) {
        if (x < 0) return -1;
        t += x;
    }
    return t;
}
