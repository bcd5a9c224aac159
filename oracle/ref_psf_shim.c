/* ref_psf_shim.c -- test infrastructure: exposes the reference's static
 * measure_tile_psf_sigma (pipeline.c:107-196) for the oracle pins. The reference source
 * is included unmodified from the reference tree (oracle/Makefile passes its path) and
 * compiled with the reference's own flags; this file adds only the exported wrapper. */
#include "pipeline.c"

double ref_measure_tile_psf_sigma(const unsigned char *vol, int Z, int Y, int X) {
    return measure_tile_psf_sigma(vol, Z, Y, X);
}
