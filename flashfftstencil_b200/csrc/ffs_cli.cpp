// Command-line driver with the reference's surface.
//
//   ffs 1d|2d|3d <shape> <size...> <T> [options]
//   1d.out|2d.out|3d.out <shape> <size...> <T> [options]   (dimension from the program name)
//
// Mirrors src/1D/1d_main.cu:32-249, src/2D/2d_main.cu:40-285, src/3D/3d_main.cu:36-194 and
// README.md:43-58: one size for every dimension or one per dimension (x first),
// `--custom` reads the (2r+1)^dim weights of the shape's footprint from stdin
// (whitespace separated, dx fastest), `--help` prints usage.  Prints the
// reference's CSV line "FlashFFTStencil, <label>, <nz>, <ny>, <nx>, <T>, <ms>, <GStencil/s>"
// (src/2D/2d_main.cu:185).  Unlike the reference, T counts true time steps and
// any size is accepted; inputs are seeded uniform[0,1) values.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include "ffs.h"

namespace {

void usage(const char *prog)
{
    std::printf(
        "Program name: FlashFFTStencil (B200)\n"
        "Usage: %s [1d|2d|3d] <stencil-shape> <input_size...> <time_steps> [options]\n"
        "  stencil-shape: Heat-1D 1D5P 1D7P | Heat-2D Box2D9P Star2D9P Box2D25P | Heat-3D Box3D27P\n"
        "  input_size:    one size for all dimensions, or one per dimension (x first)\n"
        "options:\n"
        "  --help                 this text\n"
        "  --custom               read the shape's (2r+1)^dim weights from stdin (dx fastest)\n"
        "  --weights FILE         read the weights from FILE instead\n"
        "  --boundary periodic|fixed   (default periodic, the reference's wrap)\n"
        "  --form auto|fp64_fft|fp64|ozaki|bf16x3   (default auto: the fastest FP64-exact form, fp64_fft)\n"
        "  --tau N                fused steps per pass (default: autotuned)\n"
        "  --slices N             Ozaki slice count (default: automatic)\n"
        "  --repeat N             timed repetitions (default 1, after one warm-up)\n"
        "  --seed N               input seed (default 1)\n"
        "  --json                 also print the plan as JSON\n",
        prog);
}

bool read_weights(std::istream &in, std::vector<double> &w, size_t count)
{
    w.clear();
    double v;
    while (w.size() < count && (in >> v))
        w.push_back(v);
    return w.size() == count;
}

} // namespace

int main(int argc, char **argv)
{
    std::string prog = argv[0];
    const size_t slash = prog.find_last_of('/');
    const std::string base = slash == std::string::npos ? prog : prog.substr(slash + 1);
    std::vector<std::string> pos;
    bool custom = false, json = false;
    std::string weights_file, boundary = "periodic", form = "auto";
    int tau = 0, slices = 0, repeat = 1;
    unsigned long seed = 1;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto need = [&](const char *what) -> std::string {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "%s needs a value\n", what);
                std::exit(1);
            }
            return argv[++i];
        };
        if (a == "--help" || a == "-h") {
            usage(base.c_str());
            return 0;
        } else if (a == "--custom") {
            custom = true;
        } else if (a == "--json") {
            json = true;
        } else if (a == "--weights") {
            weights_file = need("--weights");
            custom = true;
        } else if (a == "--boundary") {
            boundary = need("--boundary");
        } else if (a == "--form") {
            form = need("--form");
        } else if (a == "--tau") {
            tau = std::atoi(need("--tau").c_str());
        } else if (a == "--slices") {
            slices = std::atoi(need("--slices").c_str());
        } else if (a == "--repeat") {
            repeat = std::max(1, std::atoi(need("--repeat").c_str()));
        } else if (a == "--seed") {
            seed = std::strtoul(need("--seed").c_str(), nullptr, 10);
        } else if (a.size() > 2 && a[0] == '-' && a[1] == '-') {
            std::fprintf(stderr, "unknown option %s\n", a.c_str());
            usage(base.c_str());
            return 1;
        } else {
            pos.push_back(a);
        }
    }
    int dim = 0;
    if (base.size() >= 2 && (base[0] >= '1' && base[0] <= '3') && base[1] == 'd')
        dim = base[0] - '0';
    if (!dim && !pos.empty() && pos[0].size() == 2 && pos[0][1] == 'd' && pos[0][0] >= '1' && pos[0][0] <= '3') {
        dim = pos[0][0] - '0';
        pos.erase(pos.begin());
    }
    if (!dim || (pos.size() != 3 && pos.size() != (size_t)(dim + 2))) {
        usage(base.c_str());
        return 1;
    }
    ffs_shape shape;
    int sdim = 0, r = 0;
    const char *label = nullptr;
    if (ffs_shape_lookup(pos[0].c_str(), &shape, &sdim, &r, &label, nullptr, 0) != FFS_OK || sdim != dim) {
        std::cout << "FlashFFTStencil: unknown " << dim << "-D stencil shape '" << pos[0] << "'" << std::endl;
        return 1;
    }
    int64_t ext[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d)
        ext[d] = std::atoll(pos[pos.size() == 3 ? 1 : 1 + d].c_str());
    const int T = std::atoi(pos.back().c_str());
    size_t nw = 1;
    for (int d = 0; d < dim; ++d)
        nw *= 2 * r + 1;
    std::vector<double> w(nw);
    ffs_shape_lookup(pos[0].c_str(), nullptr, nullptr, nullptr, nullptr, w.data(), (int)w.size());
    if (custom) {
        bool ok;
        if (!weights_file.empty()) {
            std::ifstream f(weights_file);
            ok = f && read_weights(f, w, nw);
        } else {
            ok = read_weights(std::cin, w, nw);
        }
        if (!ok) {
            std::fprintf(stderr, "--custom: expected %zu weights\n", nw);
            return 1;
        }
    }
    ffs_problem p;
    std::memset(&p, 0, sizeof(p));
    p.dim = dim;
    p.shape = custom ? FFS_SHAPE_CUSTOM : shape;
    p.radius = r;
    p.weights = custom ? w.data() : nullptr;
    for (int d = 0; d < 3; ++d)
        p.extents[d] = ext[d];
    p.T = T;
    p.boundary = boundary == "fixed" ? FFS_BOUNDARY_FIXED : FFS_BOUNDARY_PERIODIC;
    if (form == "fp64" || form == "fp64_dmma")
        p.form = FFS_FORM_FP64_DMMA;
    else if (form == "fp64_fft")
        p.form = FFS_FORM_FP64_FFT;
    else if (form == "ozaki")
        p.form = FFS_FORM_OZAKI_I8;
    else if (form == "bf16x3")
        p.form = FFS_FORM_BF16X3;
    else if (form == "auto")
        p.form = FFS_FORM_AUTO;
    else {
        std::fprintf(stderr, "FlashFFTStencil: unknown --form '%s'\n", form.c_str());
        return 1;
    }
    p.slices = slices;
    p.tau = tau;
    ffs_plan *plan = nullptr;
    if (ffs_plan_create(&plan, &p) != FFS_OK) {
        std::fprintf(stderr, "FlashFFTStencil: %s\n", ffs_last_error_string());
        return 1;
    }
    const size_t cells = (size_t)ext[0] * ext[1] * ext[2];
    std::vector<double> h(cells);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    for (double &v : h)
        v = U(rng);
    double *d_in = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_in, cells * 8) != cudaSuccess || cudaMalloc(&d_out, cells * 8) != cudaSuccess) {
        std::fprintf(stderr, "FlashFFTStencil: device allocation failed\n");
        return 1;
    }
    cudaMemcpy(d_in, h.data(), cells * 8, cudaMemcpyHostToDevice);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (ffs_execute(plan, d_in, d_out, nullptr) != FFS_OK) { // warm-up
        std::fprintf(stderr, "FlashFFTStencil: %s\n", ffs_last_error_string());
        return 1;
    }
    cudaEventRecord(e0);
    for (int i = 0; i < repeat; ++i)
        ffs_execute(plan, d_in, d_out, nullptr);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        std::fprintf(stderr, "FlashFFTStencil: %s\n", cudaGetErrorString(err));
        return 1;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= repeat;
    const double gs = (double)cells * T / ms / 1e6;
    std::cout << "FlashFFTStencil, " << label << ", " << ext[2] << ", " << ext[1] << ", " << ext[0] << ", " << T
              << ", " << ms << ", " << gs << std::endl;
    if (json) {
        ffs_plan_info info;
        ffs_plan_get_info(plan, &info);
        std::printf("{\"dim\": %d, \"radius\": %d, \"form\": %d, \"tile\": %d, \"halo\": %d, \"useful\": %d, "
                    "\"tau\": %d, \"tau_last\": %d, \"passes\": %d, \"slices\": %d, \"tiles\": %lld, "
                    "\"ms\": %.6f, \"gstencil_s\": %.3f}\n",
                    info.dim, info.radius, (int)info.form, info.tile, info.halo, info.useful, info.tau,
                    info.tau_last, info.passes, info.slices, (long long)info.tiles, ms, gs);
    }
    cudaFree(d_in);
    cudaFree(d_out);
    ffs_plan_destroy(plan);
    return 0;
}
