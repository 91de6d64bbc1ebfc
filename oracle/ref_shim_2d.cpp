// Thin C-ABI shim around the reference's own 2D CPU stencil, compiled from the
// reference sources where they lie (src/2D/check_correct.hpp:17-33 rotateKernel180,
// :35-49 convertTo2D, :64-100 stencil2D).  Test infrastructure only.
#define areArraysEqual ffs_ref2d_areArraysEqual
#include "check_correct.hpp"

extern "C" void ffs_ref_stencil2d(const double *in, int width, const double *k, int K, double *out)
{
    Matrix input = convertTo2D(const_cast<double *>(in), width);
    Matrix kernel(K, std::vector<double>(K));
    for (int i = 0; i < K; ++i)
        for (int j = 0; j < K; ++j)
            kernel[i][j] = k[i * K + j];
    std::vector<double> r = stencil2D(input, kernel);
    for (int i = 0; i < width * width; ++i)
        out[i] = r[i];
}

extern "C" void ffs_ref_rotate180(const double *k, int K, double *out)
{
    std::vector<double> kv(k, k + K * K);
    Matrix r = rotateKernel180(kv);
    for (int i = 0; i < K; ++i)
        for (int j = 0; j < K; ++j)
            out[i * K + j] = r[i][j];
}
