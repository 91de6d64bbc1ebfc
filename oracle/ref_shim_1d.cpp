// Thin C-ABI shim around the reference's own 1D CPU stencil, compiled from the
// reference sources where they lie (src/1D/check_correct.hpp:15-38).  Test
// infrastructure only: used to pin the oracle and to make tests/golden fixtures.
#define areArraysEqual ffs_ref1d_areArraysEqual
#include "check_correct.hpp"

extern "C" void ffs_ref_stencil1d(const double *in, int n, const double *k, int K, double *out)
{
    stencil1D(in, n, k, K, out);
}
