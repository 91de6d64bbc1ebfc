// Host-only plan builder (no CUDA calls): shape table, FP64 spectra, DFT
// tables, tile geometry, autotuned fusion depth and fixed-boundary band boxes.
#pragma once
#include <vector_types.h>

#include <string>
#include <vector>

#include "ffs.h"
#include "ffs_kernels.h"

namespace ffst {

constexpr size_t kBandSmemLimit = 200 * 1024;

struct ShapeDef {
    const char *name;
    ffs_shape id;
    int dim;
    int radius;
    const char *label; // the reference's CSV label (src/2D/2d_main.cu:179-183 ...)
};

const ShapeDef *find_shape(const char *name);
const ShapeDef *find_shape_id(ffs_shape id);
std::vector<double> shape_weights(const ShapeDef &sd);

// One kind of fused pass (all passes but the last share kind 0).
struct PassSpec {
    int tau = 0, halo = 0, useful = 0;
    std::vector<double2> spectrum; // spectrum^tau / n^d in kernel position order
    std::vector<BandBox> boxes;    // fixed-boundary band boxes
    int64_t band_max_vol = 0;
    int64_t t0[3] = {0, 0, 0}, nt[3] = {1, 1, 1};
    int64_t vlo[3] = {0, 0, 0}, vhi[3] = {1, 1, 1};
    int64_t npx = 0, nitems = 0;
};

struct PlanSpec {
    int dim = 0, radius = 0;
    int64_t n[3] = {1, 1, 1};
    size_t cells = 0;
    std::vector<double> weights; // dense (2r+1)^dim
    std::vector<int4> taps;      // non-zero taps {dx, dy, dz, weight index}
    int T = 0;
    ffs_boundary boundary = FFS_BOUNDARY_PERIODIC;
    int open_faces = 0;          // faces that are cuts through a larger grid (no band there)
    ffs_form form = FFS_FORM_FP64_DMMA;
    int slices = 0;
    int tile = 0;
    int tau = 0, tau_last = 0, passes = 0;
    int npass_kinds = 0, last_kind = 0;
    PassSpec pass[2];
    std::vector<double2> tables;
    std::vector<unsigned char> a_slices; // tcgen05 forms: DFT-matrix slices in operand layout
    double est_seconds = 0.0; // autotuner's model estimate for all passes
};

// Validate `p`, pick form/tile/tau and fill `out`.  With `with_data` false the
// spectra and tables are not computed (fast describe path).
ffs_status build_plan_spec(const ffs_problem &p, PlanSpec *out, std::string *why, bool with_data = true);
void fill_plan_info(const PlanSpec &sp, ffs_plan_info *info);

// Model-ranked fusion depths for a problem (best first), at most `count`.
std::vector<int> tau_candidates(const ffs_problem &p, int count);

// Measured-tuning table: key of a problem class, and lookup/record of its best tau;
// slice_key names the class without its slice count, whose entry is the calibrated
// Ozaki slice count, and tile_key the class without its tile edge, whose entry is the
// measured tile edge of the 3D butterfly form (ffs_autotune).
std::string tune_key(const PlanSpec &sp);
std::string slice_key(const PlanSpec &sp);
std::string tile_key(const PlanSpec &sp);
int tune_lookup(const std::string &key);
void tune_record(const std::string &key, int value);

// Ozaki slice count of a problem without a calibrated one: 7 balanced base-256
// digits carry 54 bits, FP64-level accuracy.
constexpr int kDefaultOzakiSlices = 7;
// Calibration bound of ffs_autotune's slice choice: max relative difference to
// the FP64 form at most 1e-12 with a margin of 1.5.
constexpr double kSliceCalibrationTol = 1e-12 / 1.5;

// Modelled seconds of the host-buffer pipelines for `grids` grids: the
// whole-grid pipeline (copy-in, compute and copy-out of consecutive grids
// overlap), and the slab pipeline with per-slab copy-in a, compute b and
// copy-out c (a three-stage pipeline over grids * count items).
struct SlabModel {
    int count = 1;       // slabs per grid (1 = whole grid)
    bool forced = false; // count set by FFS_HOST_SLABS
    double a = 0, b = 0, c = 0, copy = 0, comp = 0;
    double whole(int grids) const { return 2 * copy + comp + (grids - 1) * std::max(copy, comp); }
    double slabs(int grids) const
    {
        return a + b + c + (double)(grids * count - 1) * std::max(a, std::max(b, c));
    }
};

// The problem of one slab of a grid: `rows` along the slowest axis, `open` cut
// faces, the parent's weights (which must outlive the problem), T, boundary,
// resolved form, slices and tau.
ffs_problem slab_problem(const PlanSpec &sp, int64_t rows, int open);

// Slab count and model of the host-buffer pipeline for one grid of `sp`.
SlabModel slab_model(const PlanSpec &sp);

// Records the thread's last error message (ffs_last_error_string) and returns st.
ffs_status set_error(ffs_status st, const std::string &msg);

} // namespace ffst
