// fy_spectral.cuh -- half-spectrum 3-D transform passes shared by the deconvolution and
// the phase-correlation kernels.
//
// Layout in HBM: the Hermitian half spectrum of a real (pz,py,px) volume as interleaved
// float2 rows spec[(z*py + y)*hxp + kx], kx < hx = px/2+1, row pitch hxp = hx rounded up to
// 16 complex (128 B) so every W=16 column tile is one aligned 128-byte segment per point.
// Only the planes that are actually distinct are stored: with reflect padding (deconv),
// plane z >= nz equals plane reflect(z) before the Z transform, so the buffer holds nz
// planes and the Z pass gathers the reflected planes on load; with zero padding
// (phase correlation) planes >= nz are zero and are synthesised, not read.
#pragma once
#include "fy_fft.cuh"

struct SpecGeom {
    int nz, ny, nx;   // logical volume
    int pz, py, px;   // padded transform sizes
    int hx, hxp;      // half-spectrum width and row pitch (complex elements)
    int zero_pad;     // 0: reflect padding (paganin.c:121-128), 1: zero padding (phasecorr.c:76-87)
};

// Hermitian untangle of one two-for-one line: L = FFT(a + i b) ->
//   A[k] = (L[k] + conj(L[-k]))/2,  B[k] = (L[k] - conj(L[-k]))/(2i)   (paganin.c:179-191)
FY_D void untangle(float2 L, float2 M, float2& A, float2& B) {
    A = make_float2(0.5f * (L.x + M.x), 0.5f * (L.y - M.y));
    B = make_float2(0.5f * (L.y + M.y), 0.5f * (M.x - L.x));
}

// Two half-spectrum rows A,B -> the full complex line L = a + i b for the C2R inverse
// (paganin.c:271-280): L[k] = A[k] + iB[k] (k < hx), L[px-m] = conj(A[m]) + i conj(B[m]).
FY_D float2 pack_lo(float2 A, float2 B) { return make_float2(A.x - B.y, A.y + B.x); }
FY_D float2 pack_hi(float2 A, float2 B) { return make_float2(A.x + B.y, -A.y + B.x); }
