// Host-only plan builder.  Replaces the reference's CreatePlan
// (src/1D/create_fft_pfa_plan.cu:19-228, src/2D/create_fft_pfa_plan.cu:17-147,
// src/3D/create_fft_pfa_plan.cu:17-139), which builds DFT-8 matrices with
// cos/sin and the kernel spectrum with cuFFT and uploads both to __constant__.
// Here everything is FP64 host arithmetic: the spectrum is a direct DFT of the
// (2r+1)^d taps (no cuFFT), raised to the fused step count by repeated
// squaring in extended precision, divided by n^d, and permuted into the order in
// which the tile kernel holds its frequencies.
#include "ffs_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

namespace ffst {

namespace {

const ShapeDef kShapes[] = {
    {"Heat-1D", FFS_SHAPE_HEAT_1D, 1, 1, "1d1r"},       {"1D5P", FFS_SHAPE_1D5P, 1, 2, "1d2r"},
    {"1D7P", FFS_SHAPE_1D7P, 1, 3, "1d3r"},             {"Heat-2D", FFS_SHAPE_HEAT_2D, 2, 1, "star_2d1r"},
    {"Box2D9P", FFS_SHAPE_BOX2D9P, 2, 1, "box_2d1r"},   {"Star2D9P", FFS_SHAPE_STAR2D9P, 2, 2, "star_2d2r"},
    {"Box2D25P", FFS_SHAPE_BOX2D25P, 2, 2, "box_2d2r"}, {"Heat-3D", FFS_SHAPE_HEAT_3D, 3, 1, "star_3d1r"},
    {"Box3D27P", FFS_SHAPE_BOX3D27P, 3, 1, "box_3d1r"},
};

bool iequals(const char *a, const char *b)
{
    for (; *a && *b; ++a, ++b)
        if (tolower((unsigned char)*a) != tolower((unsigned char)*b))
            return false;
    return *a == *b;
}

struct CLD { // extended-precision complex for spectrum powers
    long double re, im;
};
inline CLD mul(CLD a, CLD b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
CLD cpow(CLD z, int e)
{
    CLD r{1.0L, 0.0L};
    while (e > 0) {
        if (e & 1)
            r = mul(r, z);
        z = mul(z, z);
        e >>= 1;
    }
    return r;
}

// exp(-2 pi i m / n) for m in [0, n), computed in long double.
std::vector<CLD> roots(int n)
{
    std::vector<CLD> r(n);
    const long double two_pi = 6.283185307179586476925286766559L;
    for (int m = 0; m < n; ++m) {
        long double a = two_pi * (long double)m / (long double)n;
        r[m] = {cosl(a), -sinl(a)};
    }
    return r;
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Symbol of the correlation stencil at integer frequency k (per dim) on an n^d
// grid: S(k) = sum_d w[d] exp(+2 pi i d.k / n).
CLD symbol(const PlanSpec &sp, const std::vector<CLD> &rt, int n, const int k[3])
{
    const int r = sp.radius, K = 2 * r + 1;
    const int ry = sp.dim >= 2 ? r : 0, rz = sp.dim >= 3 ? r : 0, Ky = 2 * ry + 1;
    CLD s{0.0L, 0.0L};
    for (int dz = -rz; dz <= rz; ++dz)
        for (int dy = -ry; dy <= ry; ++dy)
            for (int dx = -r; dx <= r; ++dx) {
                const double w = sp.weights[((dz + rz) * Ky + (dy + ry)) * K + (dx + r)];
                if (w == 0.0)
                    continue;
                // exp(+2 pi i m / n) = conj(root[m]) = root[(-m) mod n]
                int64_t m = (int64_t)dx * k[0] + (int64_t)dy * k[1] + (int64_t)dz * k[2];
                m = ((-m) % n + n) % n;
                s.re += (long double)w * rt[m].re;
                s.im += (long double)w * rt[m].im;
            }
    return s;
}

// ---- per-form tile geometry ----
int tile_edge(int dim, ffs_form form)
{
    (void)form;
    switch (dim) {
    case 1:
        return 4096;
    case 2:
        return 64;
    default:
        return 16;
    }
}

// Second tile edge of the FP64 butterfly form: 128 x 128 (one real tile per CTA) in 2D,
// 32^3 (a four-CTA cluster per pair) in 3D; 0 for the forms with one edge.
int alt_tile_edge(int dim, ffs_form form)
{
    if (form != FFS_FORM_FP64_FFT)
        return 0;
    return dim == 2 ? 128 : (dim == 3 ? 32 : 0);
}

int round_even(int v) { return (v + 1) & ~1; }

// Geometry of one pass kind with fusion depth tau.
void geometry(const PlanSpec &sp, int tau, PassSpec *ps)
{
    const int n = sp.tile;
    ps->tau = tau;
    ps->halo = round_even(sp.radius * tau);
    ps->useful = n - 2 * ps->halo;
    const int64_t rt = (int64_t)sp.radius * tau;
    for (int d = 0; d < 3; ++d) {
        if (d >= sp.dim) {
            ps->vlo[d] = 0;
            ps->vhi[d] = 1;
            ps->t0[d] = 0;
            ps->nt[d] = 1;
            continue;
        }
        if (sp.boundary == FFS_BOUNDARY_PERIODIC) {
            ps->vlo[d] = 0;
            ps->vhi[d] = sp.n[d];
        } else { // cells within r*tau of a fixed face go to the band; an open face has none
            ps->vlo[d] = (sp.open_faces >> (2 * d) & 1) ? 0 : std::min<int64_t>(rt, sp.n[d]);
            ps->vhi[d] = (sp.open_faces >> (2 * d + 1) & 1) ? sp.n[d]
                                                             : std::max<int64_t>(sp.n[d] - rt, ps->vlo[d]);
        }
        ps->t0[d] = ps->vlo[d] / ps->useful;
        const int64_t t1 = ceil_div(ps->vhi[d], ps->useful);
        ps->nt[d] = std::max<int64_t>(0, t1 - ps->t0[d]);
    }
    bool empty = false;
    for (int d = 0; d < sp.dim; ++d)
        empty |= ps->vhi[d] <= ps->vlo[d];
    if (empty) {
        ps->npx = 0;
        ps->nitems = 0;
    } else {
        // tile pairs along x (re / im of one complex tile), except the 2D 128 x 128 kernel,
        // which packs row pairs of one real tile instead
        ps->npx = (sp.dim == 2 && sp.tile == 128) ? ps->nt[0] : ceil_div(ps->nt[0], 2);
        ps->nitems = ps->npx * ps->nt[1] * ps->nt[2];
    }
}

// Fixed-boundary band: every cell outside the exact window, partitioned into
// slabs (cell goes to the highest dim in which it is in the band) and boxes
// small enough that box + r*tau halo fits the band kernel's shared memory.
void band_boxes(const PlanSpec &sp, PassSpec *ps)
{
    ps->boxes.clear();
    ps->band_max_vol = 0;
    if (sp.boundary != FFS_BOUNDARY_FIXED || ps->tau == 0)
        return;
    const int64_t rt = (int64_t)sp.radius * ps->tau;
    const size_t tap_bytes = sp.taps.size() * (sizeof(int4) + sizeof(double)) + 64;
    const int64_t vol_limit = (int64_t)((kBandSmemLimit - tap_bytes) / (2 * sizeof(double)));
    for (int d = sp.dim - 1; d >= 0; --d) {
        for (int side = 0; side < 2; ++side) {
            int64_t lo[3], hi[3];
            for (int e = 0; e < 3; ++e) {
                if (e >= sp.dim) {
                    lo[e] = 0;
                    hi[e] = 1;
                } else if (e > d) {
                    lo[e] = ps->vlo[e];
                    hi[e] = ps->vhi[e];
                } else if (e < d) {
                    lo[e] = 0;
                    hi[e] = sp.n[e];
                } else if (side == 0) {
                    lo[e] = 0;
                    hi[e] = ps->vlo[e];
                } else {
                    lo[e] = ps->vhi[e];
                    hi[e] = sp.n[e];
                }
            }
            bool empty = false;
            for (int e = 0; e < 3; ++e)
                empty |= hi[e] <= lo[e];
            if (empty)
                continue;
            int64_t chunk[3];
            for (int e = 0; e < 3; ++e)
                chunk[e] = hi[e] - lo[e];
            auto staged_bound = [&]() {
                int64_t v = 1;
                for (int e = 0; e < sp.dim; ++e)
                    v *= std::min<int64_t>(chunk[e] + 2 * rt, sp.n[e]);
                return v;
            };
            // cap the long dims of a box: the band kernel runs beside the tile kernel, and its
            // CTAs hold SMs the tile CTAs then start late on.  2D: 32 (Box2D9P 4096^2, caps
            // 16 / 32 / 64 / 256 -> 826 / 849 / 831 / 657 GStencil/s; with the band launched
            // after the 128 x 128 tile kernel, caps 24 / 32 / 48 / 64 -> 955 / 990 / 918 / 918,
            // and Box2D9P 8192^2 1117 / 1124 / 1110 / 1110; on grids below 2^24 cells
            // the 512-problem mixed batch took 204.0 / 210.9 / 207.1 at 16 / 32 / 64 with the 3D
            // cap at 16).  3D: 64 on grids of 2^24 cells and more (Box3D27P 512^3, caps 16 / 64
            // -> 149.5 / 151.9), 32 below (the batch: 217.0 against 210.9 at 16, 2D cap 32).
            const bool big = sp.cells >= (size_t)1 << 24;
            const int64_t long_cap = sp.dim == 1 ? (int64_t)1 << 30 : (sp.dim == 2 ? 32 : (big ? 64 : 32));
            for (int e = 0; e < sp.dim; ++e)
                if (e != d)
                    chunk[e] = std::min(chunk[e], long_cap);
            while (staged_bound() > vol_limit) {
                int big = -1;
                for (int e = 0; e < sp.dim; ++e)
                    if (chunk[e] > 1 && (big < 0 || chunk[e] > chunk[big]))
                        big = e;
                if (big < 0)
                    break;
                chunk[big] = (chunk[big] + 1) / 2;
            }
            for (int64_t z = lo[2]; z < hi[2]; z += chunk[2])
                for (int64_t y = lo[1]; y < hi[1]; y += chunk[1])
                    for (int64_t x = lo[0]; x < hi[0]; x += chunk[0]) {
                        BandBox b;
                        const int64_t o[3] = {x, y, z};
                        int64_t vol = 1;
                        for (int e = 0; e < 3; ++e) {
                            b.lo[e] = o[e];
                            b.ext[e] = (int32_t)std::min<int64_t>(chunk[e], hi[e] - o[e]);
                            if (e < sp.dim) {
                                const int64_t L = std::max<int64_t>(o[e] - rt, 0);
                                const int64_t R = std::min<int64_t>(o[e] + b.ext[e] + rt, sp.n[e]);
                                vol *= R - L;
                            }
                        }
                        ps->band_max_vol = std::max(ps->band_max_vol, vol);
                        ps->boxes.push_back(b);
                    }
        }
    }
}

// One 32^3 complex tile pair on a four-SM cluster (FP64 butterflies), measured: 27-33 us
// per pair on Box3D27P 512^3 (2.97 ms for 3610 pairs at tau 2, 5.25 ms for 5324 at tau 4),
// with 33 clusters resident on 148 SMs.  The pair holds ten times the butterfly work of a
// 16^3 pair, but a CTA of 32-point lines runs 8 warps per SM against 24.
constexpr double kTile32PairSeconds = 30e-6;
constexpr double kTile32ClustersPerSm = 33.0 / 148.0;

// One 128 x 128 real tile on one SM (FP64 butterflies), measured: 20 us (Box2D9P 4096^2,
// tau 16: 0.251-0.257 ms for 1849 tiles, 12.5 per SM), against 5.8 us for a 64 x 64 pair.
constexpr double kTile128Seconds = 20e-6;

// Model of one pass in seconds (used to pick tau).  Rough per-form constants;
// the tile cost is the measured order of one tile pair per SM.
double pass_cost(const PlanSpec &sp, const PassSpec &ps, int num_sms)
{
    double tile_pair_s = 12e-6; // one 64x64 (2D) or 4096 (1D) complex tile pair on one SM (FP64 DMMA)
    if (sp.dim == 3)
        tile_pair_s = 10e-6;
    if (sp.form == FFS_FORM_OZAKI_I8)
        tile_pair_s = 4e-6 * sp.slices;
    else if (sp.form == FFS_FORM_FP64_FFT)
        tile_pair_s = sp.dim == 3 ? 3e-6 : (sp.dim == 2 ? 5.7e-6 : 6e-6); // 2D: 0.142 ms for 3698 pairs, 25 per SM
    else if (sp.form == FFS_FORM_BF16X3)
        tile_pair_s = 6e-6;
    // the 32^3 tile: one pair per four-SM cluster at a time
    const bool cluster = sp.dim == 3 && sp.tile == 32;
    if (cluster)
        tile_pair_s = kTile32PairSeconds;
    if (sp.dim == 2 && sp.tile == 128)
        tile_pair_s = kTile128Seconds;
    const double waves = std::ceil((double)ps.nitems / (cluster ? std::floor(kTile32ClustersPerSm * num_sms) : num_sms));
    // band boxes run concurrently, several per SM; a box costs its direct
    // stepping work plus a per-step barrier latency
    double box_max = 0.0, box_sum = 0.0;
    for (const BandBox &b : ps.boxes) {
        double v = 1.0;
        for (int e = 0; e < sp.dim; ++e)
            v *= std::min<double>(b.ext[e] + 2.0 * sp.radius * ps.tau, (double)sp.n[e]);
        const double bt = v * ps.tau * (double)sp.taps.size() / 60e9 + ps.tau * 0.3e-6;
        box_max = std::max(box_max, bt);
        box_sum += bt;
    }
    const double band = ps.boxes.empty() ? 0.0 : std::max(box_max, box_sum / (num_sms * 4.0)) + 3e-6;
    return waves * tile_pair_s + band + 4e-6;
}

int max_tau(const PlanSpec &sp)
{
    const int n = sp.tile;
    const int r = sp.radius;
    int tau_max = sp.T;
    if (r > 0)
        tau_max = std::min(tau_max, (n - 8) / 2 / r); // keep u >= 8
    tau_max = std::max(tau_max, 1);
    if (r > 0) // halo is rounded up to even: make sure u stays >= 8
        while (tau_max > 1 && n - 2 * round_even(r * tau_max) < 8)
            --tau_max;
    return tau_max;
}

double model_cost(const PlanSpec &sp, int tau)
{
    PassSpec ps;
    geometry(sp, tau, &ps);
    band_boxes(sp, &ps);
    const int passes = (sp.T + tau - 1) / tau;
    return passes * pass_cost(sp, ps, 148);
}

void pick_tau(PlanSpec *sp, int tau_override)
{
    const int n = sp->tile;
    const int r = sp->radius;
    int tau_max = sp->T;
    if (r > 0)
        tau_max = std::min(tau_max, (n - 8) / 2 / r); // keep u >= 8
    tau_max = std::max(tau_max, 1);
    if (r > 0) // halo is rounded up to even: make sure u stays >= 8
        while (tau_max > 1 && n - 2 * round_even(r * tau_max) < 8)
            --tau_max;
    int best = tau_override > 0 ? std::min(tau_override, tau_max) : 0;
    if (!best) { // a measured choice for this problem class wins over the model
        const int tuned = tune_lookup(tune_key(*sp));
        if (tuned > 0 && tuned <= tau_max)
            best = tuned;
    }
    if (!best) {
        double best_cost = 1e300;
        for (int tau = 1; tau <= tau_max; ++tau) {
            PassSpec ps;
            geometry(*sp, tau, &ps);
            band_boxes(*sp, &ps);
            const int passes = (sp->T + tau - 1) / tau;
            const double c = passes * pass_cost(*sp, ps, 148);
            if (c < best_cost * (1 - 1e-9)) {
                best_cost = c;
                best = tau;
            }
        }
    }
    sp->tau = best;
    sp->passes = (sp->T + best - 1) / best;
    sp->tau_last = sp->T - (sp->passes - 1) * best;
}

// Tile edge of the 3D butterfly form: the autotuner's measured choice for the problem
// class when it has one, else the edge whose best modelled solve is shorter.
int pick_tile(const PlanSpec &sp, int tau_override)
{
    const int tuned = tune_lookup(tile_key(sp));
    const int edges[2] = {tile_edge(sp.dim, sp.form), alt_tile_edge(sp.dim, sp.form)};
    const int tuned_ok = tuned == edges[0] || tuned == edges[1];
    if (tuned_ok)
        return tuned;
    int best = edges[0];
    double best_cost = 1e300;
    for (int tile : edges) {
        PlanSpec t = sp;
        t.tile = tile;
        pick_tau(&t, tau_override);
        const double c = model_cost(t, t.tau);
        if (c < best_cost * (1 - 1e-9)) {
            best_cost = c;
            best = tile;
        }
    }
    return best;
}

void make_spectrum_2d(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 64;
    const auto rt = roots(n);
    out->resize(n * n);
    const long double scale = 1.0L / (n * n);
    // position p holds frequency (p >> 3) + 8 * (p & 7) (two radix-8 stages)
    for (int px = 0; px < n; ++px)
        for (int py = 0; py < n; ++py) {
            const int k[3] = {(px >> 3) + 8 * (px & 7), (py >> 3) + 8 * (py & 7), 0};
            CLD s = cpow(symbol(sp, rt, n, k), tau);
            (*out)[px * n + py] = make_double2((double)(s.re * scale), (double)(s.im * scale));
        }
}

// 1D tile of 4096 = 64 x 64 (j = 64a + b): SMEM column position px holds the
// first-stage frequency k1 = k(px), row position py the second-stage k2 = k(py),
// k(p) = (p >> 3) + 8 * (p & 7); full frequency k1 + 64 * k2.
void make_spectrum_1d(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 4096;
    const auto rt = roots(n);
    out->resize(n);
    const long double scale = 1.0L / n;
    for (int px = 0; px < 64; ++px)
        for (int py = 0; py < 64; ++py) {
            const int k1 = (px >> 3) + 8 * (px & 7), k2 = (py >> 3) + 8 * (py & 7);
            const int k[3] = {k1 + 64 * k2, 0, 0};
            CLD s = cpow(symbol(sp, rt, n, k), tau);
            (*out)[px * 64 + py] = make_double2((double)(s.re * scale), (double)(s.im * scale));
        }
}

// 1D butterfly form: the Hermitian half k = 0..2048 at slot k + (k >> 6) (2088 slots); the
// kernel takes k > 2048 as conj S[4096 - k].
void make_spectrum_1d_half(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 4096;
    const auto rt = roots(n);
    out->assign(2088, make_double2(0.0, 0.0));
    const long double scale = 1.0L / n;
    for (int f = 0; f <= n / 2; ++f) {
        const int k[3] = {f, 0, 0};
        CLD s = cpow(symbol(sp, rt, n, k), tau);
        (*out)[f + (f >> 6)] = make_double2((double)(s.re * scale), (double)(s.im * scale));
    }
}

// tcgen05 forms: natural frequency order spec[ky * 64 + kx].
void make_spectrum_2d_natural(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 64;
    const auto rt = roots(n);
    out->resize(n * n);
    const long double scale = 1.0L / (n * n);
    for (int ky = 0; ky < n; ++ky)
        for (int kx = 0; kx < n; ++kx) {
            const int k[3] = {kx, ky, 0};
            CLD s = cpow(symbol(sp, rt, n, k), tau);
            (*out)[ky * n + kx] = make_double2((double)(s.re * scale), (double)(s.im * scale));
        }
}

// Butterfly form: the half kx = 0..32, spec[ky * 33 + kx].  Real weights make the
// symbol Hermitian, S(-k) = conj S(k), so the kernel takes kx > 32 as
// conj spec[(-ky mod 64) * 33 + 64 - kx].
void make_spectrum_2d_half(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 64, h = n / 2 + 1;
    const auto rt = roots(n);
    out->resize(n * h);
    const long double scale = 1.0L / (n * n);
    for (int ky = 0; ky < n; ++ky)
        for (int kx = 0; kx < h; ++kx) {
            const int k[3] = {kx, ky, 0};
            CLD s = cpow(symbol(sp, rt, n, k), tau);
            (*out)[ky * h + kx] = make_double2((double)(s.re * scale), (double)(s.im * scale));
        }
}

// 2D butterfly form on the 128 x 128 tile: the half kx = 0..64, spec[kx * 128 + ky] (a
// column's group reads consecutive ky).
void make_spectrum_2d128(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 128;
    const auto rt = roots(n);
    out->resize((n / 2 + 1) * n);
    const long double scale = 1.0L / (n * n);
    for (int kx = 0; kx <= n / 2; ++kx)
        for (int ky = 0; ky < n; ++ky) {
            const int k[3] = {kx, ky, 0};
            CLD s = cpow(symbol(sp, rt, n, k), tau);
            (*out)[kx * n + ky] = make_double2((double)(s.re * scale), (double)(s.im * scale));
        }
}

// 3D butterfly form: the half kx = 0..8, spec[(kx * 16 + kz) * 16 + ky] (the 32 lines
// (kz, ky) of a warp read 32 consecutive entries per kx); the kernel takes kx > 8 as
// conj spec[(16 - kx, -kz mod 16, -ky mod 16)] (Hermitian symbol).
void make_spectrum_3d_half(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 16, h = n / 2 + 1;
    const auto rt = roots(n);
    out->resize(n * n * h);
    const long double scale = 1.0L / (n * n * n);
    for (int kz = 0; kz < n; ++kz)
        for (int ky = 0; ky < n; ++ky)
            for (int kx = 0; kx < h; ++kx) {
                const int k[3] = {kx, ky, kz};
                CLD s = cpow(symbol(sp, rt, n, k), tau);
                (*out)[(kx * n + kz) * n + ky] = make_double2((double)(s.re * scale), (double)(s.im * scale));
            }
}

// 3D (the other forms): natural frequency order spec[(kz * 16 + ky) * 16 + kx].
void make_spectrum_3d_natural(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 16;
    const auto rt = roots(n);
    out->resize(n * n * n);
    const long double scale = 1.0L / (n * n * n);
    for (int kz = 0; kz < n; ++kz)
        for (int ky = 0; ky < n; ++ky)
            for (int kx = 0; kx < n; ++kx) {
                const int k[3] = {kx, ky, kz};
                CLD s = cpow(symbol(sp, rt, n, k), tau);
                (*out)[(kz * n + ky) * n + kx] = make_double2((double)(s.re * scale), (double)(s.im * scale));
            }
}

// 3D butterfly form on the 32^3 tile: natural order spec[(kz * 32 + ky) * 32 + kx] (the
// cluster kernel reads it along kx, coalesced, for its y lines).
void make_spectrum_3d32(const PlanSpec &sp, int tau, std::vector<double2> *out)
{
    const int n = 32;
    const auto rt = roots(n);
    out->resize(n * n * n);
    const long double scale = 1.0L / (n * n * n);
    for (int kz = 0; kz < n; ++kz)
        for (int ky = 0; ky < n; ++ky)
            for (int kx = 0; kx < n; ++kx) {
                const int k[3] = {kx, ky, kz};
                CLD s = cpow(symbol(sp, rt, n, k), tau);
                (*out)[(kz * n + ky) * n + kx] = make_double2((double)(s.re * scale), (double)(s.im * scale));
            }
}

// Byte offset of (row r, K byte kb) in a K-major no-swizzle tcgen05 operand with KB bytes per row.
size_t operand_offset(int r, int kb, int KB) { return (size_t)(r / 8) * (8 * KB) + (kb / 16) * 128 + (r % 8) * 16 + kb % 16; }

uint16_t bf16_rn(float f) // round to nearest even
{
    uint32_t u;
    memcpy(&u, &f, 4);
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}

float bf16_to_f(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// Balanced base-256 digits of y (|y| <= 64), most significant first: y * 256^(S-1)
// rounded once (exact in long double's 64-bit significand for S <= 8), biased by
// 0x80 per byte so that byte S-1-i is digit i + 128 (the device's digit_bytes).
static void ozaki_digits(long double y, int S, int8_t *d)
{
    const int64_t X = (int64_t)nearbyintl(ldexpl(y, 8 * (S - 1)));
    const uint64_t U = (uint64_t)X + (0x8080808080808080ull >> (8 * (8 - S)));
    for (int i = 0; i < S; ++i)
        d[i] = (int8_t)((int)((U >> (8 * (S - 1 - i))) & 255) - 128);
}

// Real-block DFT-64 matrix with interleaved rows (m = 2f + part), 128 x 128:
// A[2f][x] = Re F, A[2f][64+x] = -Im F, A[2f+1][x] = Im F, A[2f+1][64+x] = Re F, F = w64^(f x).
// Ozaki: `slices` balanced base-256 digits of the entry * 2^6; BF16: hi/mid/lo pieces.
void make_a_slices(PlanSpec *sp)
{
    const auto r64 = roots(64);
    auto entry = [&](int m, int k) -> long double {
        const int f = m >> 1, part = m & 1, half = k >> 6, x = k & 63;
        const CLD w = r64[(f * x) % 64];
        if (part == 0)
            return half == 0 ? w.re : -w.im;
        return half == 0 ? w.im : w.re;
    };
    const int S = sp->slices;
    if (sp->form == FFS_FORM_OZAKI_I8) {
        const int KB = 128, slice = 128 * KB;
        sp->a_slices.assign((size_t)S * slice, 0);
        for (int m = 0; m < 128; ++m)
            for (int k = 0; k < 128; ++k) {
                int8_t d[8];
                ozaki_digits(entry(m, k) * 64.0L, S, d);
                for (int i = 0; i < S; ++i)
                    sp->a_slices[(size_t)i * slice + operand_offset(m, k, KB)] = (unsigned char)d[i];
            }
    } else {
        const int KB = 256, slice = 128 * KB;
        sp->a_slices.assign((size_t)S * slice, 0);
        for (int m = 0; m < 128; ++m)
            for (int k = 0; k < 128; ++k) {
                double r = (double)entry(m, k);
                for (int i = 0; i < S; ++i) {
                    const uint16_t h = bf16_rn((float)r);
                    r -= (double)bf16_to_f(h);
                    memcpy(&sp->a_slices[(size_t)i * slice + operand_offset(m, 2 * k, KB)], &h, 2);
                }
            }
    }
}

// DFT-16 operand of the 3D tcgen05 forms: row n = 32 i + 2 f + part of slice i,
// K element k = 2 x + part_in:  [2f][2x] = Re F, [2f][2x+1] = -Im F,
// [2f+1][2x] = Im F, [2f+1][2x+1] = Re F, F = w16^(f x).  Ozaki: digits of F * 2^6
// (32-byte rows, slices stacked along N); BF16: hi/mid/lo pieces (64-byte rows).
void make_f16_slices(PlanSpec *sp)
{
    const auto r16 = roots(16);
    auto entry = [&](int m, int k) -> long double {
        const int f = m >> 1, po = m & 1, x = k >> 1, pi = k & 1;
        const CLD w = r16[(f * x) % 16];
        if (po == 0)
            return pi == 0 ? w.re : -w.im;
        return pi == 0 ? w.im : w.re;
    };
    const int S = sp->slices;
    if (sp->form == FFS_FORM_OZAKI_I8) {
        const int KB = 32;
        sp->a_slices.assign((size_t)S * 32 * KB, 0);
        for (int m = 0; m < 32; ++m)
            for (int k = 0; k < 32; ++k) {
                int8_t d[8];
                ozaki_digits(entry(m, k) * 64.0L, S, d);
                for (int i = 0; i < S; ++i)
                    sp->a_slices[operand_offset(32 * i + m, k, KB)] = (unsigned char)d[i];
            }
    } else {
        const int KB = 64, slice = 32 * KB;
        sp->a_slices.assign((size_t)S * slice, 0);
        for (int m = 0; m < 32; ++m)
            for (int k = 0; k < 32; ++k) {
                double r = (double)entry(m, k);
                for (int i = 0; i < S; ++i) {
                    const uint16_t h = bf16_rn((float)r);
                    r -= (double)bf16_to_f(h);
                    memcpy(&sp->a_slices[(size_t)i * slice + operand_offset(m, 2 * k, KB)], &h, 2);
                }
            }
    }
}

void make_tables(PlanSpec *sp)
{
    sp->tables.clear();
    auto push = [&](const std::vector<CLD> &r, int count) {
        for (int i = 0; i < count; ++i)
            sp->tables.push_back(make_double2((double)r[i % r.size()].re, (double)r[i % r.size()].im));
    };
    if (sp->dim == 3) { // 16th roots (radix-4 DFT matrices and twiddles)
        push(roots(16), 16);
        return;
    }
    push(roots(8), 8);
    push(roots(64), 64);
    if (sp->dim == 2 && sp->tile == 128) // the 128 x 128 kernel's twiddles w128^m
        push(roots(128), 128);
    if (sp->dim == 1) { // four-step twiddles w4096^m (m < 448) and w512^m (m < 512)
        push(roots(4096), 448);
        push(roots(512), 512);
    }
}

std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
bool g_tune_loaded = false;

void tune_load_locked()
{
    if (g_tune_loaded)
        return;
    g_tune_loaded = true;
    const char *path = getenv("FFS_TUNE_CACHE");
    if (!path)
        return;
    FILE *f = fopen(path, "r");
    if (!f)
        return;
    char key[512];
    int tau;
    while (fscanf(f, "%511s %d", key, &tau) == 2)
        g_tune[key] = tau;
    fclose(f);
}

} // namespace

// Problem class: form, slice count, tile edge, dimension, taps, boundary, T and the
// log2 size of each extent.
std::string tune_key(const PlanSpec &sp)
{
    char buf[256];
    int lg[3];
    for (int d = 0; d < 3; ++d)
        lg[d] = (int)std::lround(std::log2((double)sp.n[d]));
    snprintf(buf, sizeof(buf), "f%d.s%d.t%d.d%d.r%d.k%zu.b%d.o%d.T%d.n%d_%d_%d", (int)sp.form, sp.slices, sp.tile,
             sp.dim, sp.radius, sp.taps.size(), (int)sp.boundary, sp.open_faces, sp.T, lg[0], lg[1], lg[2]);
    return buf;
}

// The same class without the tile edge: key of the measured tile choice of the 3D
// butterfly form.
std::string tile_key(const PlanSpec &sp)
{
    char buf[256];
    int lg[3];
    for (int d = 0; d < 3; ++d)
        lg[d] = (int)std::lround(std::log2((double)sp.n[d]));
    snprintf(buf, sizeof(buf), "E.f%d.d%d.r%d.k%zu.b%d.o%d.T%d.n%d_%d_%d", (int)sp.form, sp.dim, sp.radius,
             sp.taps.size(), (int)sp.boundary, sp.open_faces, sp.T, lg[0], lg[1], lg[2]);
    return buf;
}

// The same class without the slice count: key of the calibrated Ozaki slice count.
std::string slice_key(const PlanSpec &sp)
{
    char buf[256];
    int lg[3];
    for (int d = 0; d < 3; ++d)
        lg[d] = (int)std::lround(std::log2((double)sp.n[d]));
    snprintf(buf, sizeof(buf), "S.f%d.d%d.r%d.k%zu.b%d.o%d.T%d.n%d_%d_%d", (int)sp.form, sp.dim, sp.radius,
             sp.taps.size(), (int)sp.boundary, sp.open_faces, sp.T, lg[0], lg[1], lg[2]);
    return buf;
}

int tune_lookup(const std::string &key)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(key);
    return it == g_tune.end() ? 0 : it->second;
}

void tune_record(const std::string &key, int tau)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    g_tune[key] = tau;
    if (const char *path = getenv("FFS_TUNE_CACHE")) {
        if (FILE *f = fopen(path, "a")) {
            fprintf(f, "%s %d\n", key.c_str(), tau);
            fclose(f);
        }
    }
}

std::vector<int> tau_candidates(const ffs_problem &p, int count)
{
    ffs_problem q = p;
    q.tau = 1;
    PlanSpec sp;
    std::string why;
    if (build_plan_spec(q, &sp, &why, false) != FFS_OK || sp.T == 0)
        return {};
    std::vector<std::pair<double, int>> c;
    const int tmax = max_tau(sp);
    for (int tau = 1; tau <= tmax; ++tau)
        c.push_back({model_cost(sp, tau), tau});
    std::sort(c.begin(), c.end());
    std::vector<int> out;
    for (int i = 0; i < (int)c.size() && i < count; ++i)
        out.push_back(c[i].second);
    return out;
}

const ShapeDef *find_shape(const char *name)
{
    if (!name)
        return nullptr;
    for (const ShapeDef &s : kShapes)
        if (iequals(s.name, name))
            return &s;
    return nullptr;
}

const ShapeDef *find_shape_id(ffs_shape id)
{
    for (const ShapeDef &s : kShapes)
        if (s.id == id)
            return &s;
    return nullptr;
}

// Default weights, each normalised to sum 1 (Heat-1D is (0.25, 0.5, 0.25)).
std::vector<double> shape_weights(const ShapeDef &sd)
{
    const int r = sd.radius, K = 2 * r + 1;
    int vol = 1;
    for (int d = 0; d < sd.dim; ++d)
        vol *= K;
    std::vector<double> w(vol, 0.0);
    auto at = [&](int dx, int dy, int dz) -> double & {
        const int ry = sd.dim >= 2 ? r : 0, rz = sd.dim >= 3 ? r : 0, Ky = 2 * ry + 1;
        return w[((dz + rz) * Ky + (dy + ry)) * K + (dx + r)];
    };
    switch (sd.id) {
    case FFS_SHAPE_HEAT_1D:
        w = {0.25, 0.5, 0.25};
        break;
    case FFS_SHAPE_1D5P:
        w = {0.1, 0.2, 0.4, 0.2, 0.1};
        break;
    case FFS_SHAPE_1D7P:
        w = {0.05, 0.1, 0.15, 0.4, 0.15, 0.1, 0.05};
        break;
    case FFS_SHAPE_HEAT_2D:
        at(0, 0, 0) = 0.5;
        at(1, 0, 0) = at(-1, 0, 0) = at(0, 1, 0) = at(0, -1, 0) = 0.125;
        break;
    case FFS_SHAPE_BOX2D9P:
        for (double &v : w)
            v = 0.1;
        at(0, 0, 0) = 0.2;
        break;
    case FFS_SHAPE_STAR2D9P:
        at(0, 0, 0) = 0.2;
        at(1, 0, 0) = at(-1, 0, 0) = at(0, 1, 0) = at(0, -1, 0) = 0.125;
        at(2, 0, 0) = at(-2, 0, 0) = at(0, 2, 0) = at(0, -2, 0) = 0.075;
        break;
    case FFS_SHAPE_BOX2D25P:
        for (double &v : w)
            v = 0.04;
        break;
    case FFS_SHAPE_HEAT_3D:
        at(0, 0, 0) = 0.4;
        at(1, 0, 0) = at(-1, 0, 0) = at(0, 1, 0) = at(0, -1, 0) = at(0, 0, 1) = at(0, 0, -1) = 0.1;
        break;
    case FFS_SHAPE_BOX3D27P:
        for (double &v : w)
            v = 0.9 / 26.0;
        at(0, 0, 0) = 0.1;
        break;
    default:
        break;
    }
    return w;
}

ffs_status build_plan_spec(const ffs_problem &p, PlanSpec *out, std::string *why, bool with_data)
{
    PlanSpec sp;
    auto bad = [&](ffs_status st, const std::string &m) {
        *why = m;
        return st;
    };
    for (int i = 0; i < 6; ++i)
        if (p.reserved[i] != 0)
            return bad(FFS_ERR_INVALID_ARGUMENT, "ffs_problem.reserved must be zero");
    if (p.open_faces < 0 || p.open_faces >= (1 << (2 * std::max(1, std::min(p.dim, 3)))))
        return bad(FFS_ERR_INVALID_ARGUMENT, "open_faces names a face the grid does not have");
    sp.open_faces = p.open_faces;
    if (p.dim < 1 || p.dim > 3)
        return bad(FFS_ERR_INVALID_ARGUMENT, "dim must be 1, 2 or 3");
    sp.dim = p.dim;
    if (p.shape != FFS_SHAPE_CUSTOM) {
        const ShapeDef *sd = find_shape_id(p.shape);
        if (!sd)
            return bad(FFS_ERR_INVALID_ARGUMENT, "unknown shape id");
        if (sd->dim != p.dim)
            return bad(FFS_ERR_INVALID_ARGUMENT, std::string("shape ") + sd->name + " is " +
                                                     std::to_string(sd->dim) + "-D");
        sp.radius = sd->radius;
        sp.weights = shape_weights(*sd);
    } else {
        if (p.radius < 0 || p.radius > 8)
            return bad(FFS_ERR_INVALID_ARGUMENT, "custom radius must be in [0, 8]");
        if (!p.weights)
            return bad(FFS_ERR_INVALID_ARGUMENT, "custom shape needs weights");
        sp.radius = p.radius;
    }
    const int K = 2 * sp.radius + 1;
    size_t nw = 1;
    for (int d = 0; d < p.dim; ++d)
        nw *= K;
    if (p.weights) {
        sp.weights.assign(p.weights, p.weights + nw);
        for (double v : sp.weights)
            if (!std::isfinite(v))
                return bad(FFS_ERR_INVALID_ARGUMENT, "weights must be finite");
    }
    if (sp.weights.size() != nw)
        return bad(FFS_ERR_INTERNAL, "weights size mismatch");
    for (int d = 0; d < 3; ++d) {
        const int64_t e = p.extents[d];
        if (d < p.dim && e < 1)
            return bad(FFS_ERR_INVALID_ARGUMENT, "extents must be >= 1");
        if (d >= p.dim && e != 1 && e != 0)
            return bad(FFS_ERR_INVALID_ARGUMENT, "unused extents must be 1");
        sp.n[d] = d < p.dim ? e : 1;
    }
    if (sp.n[0] > (1ll << 31) || sp.n[1] > (1ll << 31) || sp.n[2] > (1ll << 31))
        return bad(FFS_ERR_INVALID_ARGUMENT, "extent too large");
    sp.cells = (size_t)sp.n[0] * sp.n[1] * sp.n[2];
    if (p.T < 0)
        return bad(FFS_ERR_INVALID_ARGUMENT, "T must be >= 0");
    sp.T = p.T;
    if (p.boundary != FFS_BOUNDARY_PERIODIC && p.boundary != FFS_BOUNDARY_FIXED)
        return bad(FFS_ERR_INVALID_ARGUMENT, "unknown boundary");
    sp.boundary = p.boundary;
    if (p.tau < 0)
        return bad(FFS_ERR_INVALID_ARGUMENT, "tau must be >= 0");
    switch (p.form) {
    case FFS_FORM_AUTO: // the fastest FP64-exact form: the butterfly kernels
    case FFS_FORM_FP64_DMMA:
        sp.form = p.form == FFS_FORM_AUTO ? FFS_FORM_FP64_FFT : FFS_FORM_FP64_DMMA;
        if (p.slices != 0)
            return bad(FFS_ERR_INVALID_ARGUMENT, "slices only apply to the Ozaki and BF16 forms");
        break;
    case FFS_FORM_FP64_FFT:
        sp.form = FFS_FORM_FP64_FFT;
        if (p.slices != 0)
            return bad(FFS_ERR_INVALID_ARGUMENT, "slices only apply to the Ozaki and BF16 forms");
        break;
    case FFS_FORM_OZAKI_I8:
        sp.form = FFS_FORM_OZAKI_I8;
        sp.slices = p.slices; // 0: the calibrated count of the problem class, else the default (below)
        if (p.slices != 0 && (p.slices < 4 || p.slices > 8))
            return bad(FFS_ERR_INVALID_ARGUMENT, "Ozaki slices must be in [4, 8]");
        break;
    case FFS_FORM_BF16X3:
        sp.form = FFS_FORM_BF16X3;
        sp.slices = p.slices == 0 ? 3 : p.slices;
        if (sp.slices < 2 || sp.slices > 3)
            return bad(FFS_ERR_INVALID_ARGUMENT, "BF16 split count must be 2 or 3");
        break;
    default:
        return bad(FFS_ERR_INVALID_ARGUMENT, "unknown form");
    }
    if ((sp.form == FFS_FORM_OZAKI_I8 || sp.form == FFS_FORM_BF16X3) && p.dim == 1)
        return bad(FFS_ERR_UNSUPPORTED, "the Ozaki and BF16 tensor-core forms are available for 2-D and 3-D grids");
    // taps (non-zero weights) for the band kernel
    {
        const int r = sp.radius;
        const int ry = sp.dim >= 2 ? r : 0, rz = sp.dim >= 3 ? r : 0, Ky = 2 * ry + 1;
        for (int dz = -rz; dz <= rz; ++dz)
            for (int dy = -ry; dy <= ry; ++dy)
                for (int dx = -r; dx <= r; ++dx) {
                    const int idx = ((dz + rz) * Ky + (dy + ry)) * K + (dx + r);
                    if (sp.weights[idx] != 0.0)
                        sp.taps.push_back(make_int4(dx, dy, dz, idx));
                }
    }
    if (sp.form == FFS_FORM_OZAKI_I8 && sp.slices == 0) { // a calibrated count for this class wins
        const int tuned = tune_lookup(slice_key(sp));
        sp.slices = (tuned >= 4 && tuned <= 8) ? tuned : kDefaultOzakiSlices;
    }
    const int fixed_tile = tile_edge(sp.dim, sp.form);
    const int alt = alt_tile_edge(sp.dim, sp.form); // 0: the form has one edge
    if (p.tile != 0 && p.tile != fixed_tile && !(alt && p.tile == alt))
        return bad(FFS_ERR_UNSUPPORTED, "tile edge not available for this form (1D 4096, 2D 64, 3D 16; the FP64 "
                                        "butterfly form also 128 in 2D and 32 in 3D)");
    sp.tile = p.tile != 0 ? p.tile : fixed_tile;
    if (p.tile == 0 && alt && sp.T > 0)
        sp.tile = pick_tile(sp, p.tau);
    if (sp.T == 0) {
        sp.passes = 0;
        sp.npass_kinds = 0;
        *out = std::move(sp);
        return FFS_OK;
    }
    pick_tau(&sp, p.tau);
    if (sp.radius > 0 && sp.tile - 2 * round_even(sp.radius * sp.tau) < 8)
        return bad(FFS_ERR_UNSUPPORTED, "stencil radius too large for the tile");
    sp.npass_kinds = (sp.tau_last != sp.tau) ? 2 : 1;
    sp.last_kind = sp.npass_kinds - 1;
    sp.est_seconds = 0.0;
    for (int k = 0; k < sp.npass_kinds; ++k) {
        const int tau = k == 0 ? sp.tau : sp.tau_last;
        geometry(sp, tau, &sp.pass[k]);
        band_boxes(sp, &sp.pass[k]);
        if (sp.pass[k].band_max_vol > 0 &&
            band_smem_bytes(sp.pass[k].band_max_vol, (int)sp.taps.size()) > kBandSmemLimit)
            return bad(FFS_ERR_UNSUPPORTED, "fixed-boundary band does not fit shared memory at this tau");
        if (with_data) {
            if (sp.dim == 1 && sp.form == FFS_FORM_FP64_FFT)
                make_spectrum_1d_half(sp, tau, &sp.pass[k].spectrum);
            else if (sp.dim == 1)
                make_spectrum_1d(sp, tau, &sp.pass[k].spectrum);
            else if (sp.dim == 2 && sp.form == FFS_FORM_FP64_FFT && sp.tile == 128)
                make_spectrum_2d128(sp, tau, &sp.pass[k].spectrum);
            else if (sp.dim == 2 && sp.form == FFS_FORM_FP64_FFT)
                make_spectrum_2d_half(sp, tau, &sp.pass[k].spectrum);
            else if (sp.dim == 2 && sp.form != FFS_FORM_FP64_DMMA)
                make_spectrum_2d_natural(sp, tau, &sp.pass[k].spectrum);
            else if (sp.dim == 2)
                make_spectrum_2d(sp, tau, &sp.pass[k].spectrum);
            else if (sp.form == FFS_FORM_FP64_FFT && sp.tile == 32)
                make_spectrum_3d32(sp, tau, &sp.pass[k].spectrum);
            else if (sp.form == FFS_FORM_FP64_FFT)
                make_spectrum_3d_half(sp, tau, &sp.pass[k].spectrum);
            else
                make_spectrum_3d_natural(sp, tau, &sp.pass[k].spectrum);
        }
        const int count = k == 0 ? sp.passes - 1 : 1;
        sp.est_seconds += (sp.npass_kinds == 1 ? sp.passes : count) * pass_cost(sp, sp.pass[k], 148);
    }
    if (with_data) {
        make_tables(&sp);
        if (sp.form == FFS_FORM_OZAKI_I8 || sp.form == FFS_FORM_BF16X3) {
            if (sp.dim == 2)
                make_a_slices(&sp);
            else
                make_f16_slices(&sp);
        }
    }
    *out = std::move(sp);
    return FFS_OK;
}

// Sustained host<->device copy rate of one direction while the other is busy
// (pinned memory, PCIe Gen5 x16), for the slab-count model only.
constexpr double kCopyBytesPerSecond = 48e9;
// Fixed cost of one pass of a slab's sub-plan beyond the modelled tile waves:
// launches, the band kernel's latency (about 30 us for tau = 8 whatever the box
// count), and the first and last waves of a launch of a few hundred tiles.
// Measured on Box2D9P slabs of 4096 x 192..1024 cells, tau 8.
constexpr double kSlabPassSeconds = 25e-6;
constexpr int kMaxSlabs = 16;
constexpr int64_t kMinSlabBytes = 4ll << 20;

ffs_problem slab_problem(const PlanSpec &sp, int64_t rows, int open)
{
    ffs_problem q{};
    q.dim = sp.dim;
    q.shape = FFS_SHAPE_CUSTOM;
    q.radius = sp.radius;
    for (int d = 0; d < 3; ++d)
        q.extents[d] = sp.n[d];
    q.extents[sp.dim - 1] = rows;
    q.weights = sp.weights.data();
    q.T = sp.T;
    q.boundary = sp.boundary;
    q.form = sp.form;
    q.slices = sp.slices;
    q.tau = sp.tau;
    q.tile = sp.tile; // the whole grid's tile edge and fused step count
    q.open_faces = open;
    return q;
}

// Slab count for one grid (1 = whole grid).  The environment variable
// FFS_HOST_SLABS forces a count (1 disables the slab path).  Otherwise slabs
// are at least 4 r T rows (ghost rows at most half the stepped rows) and 4 MiB,
// at most 16, and the count with the smallest modelled time wins.
SlabModel slab_model(const PlanSpec &sp)
{
    SlabModel m;
    if (sp.dim < 2 || sp.passes == 0 || sp.open_faces != 0 ||
        (sp.boundary != FFS_BOUNDARY_FIXED && sp.boundary != FFS_BOUNDARY_PERIODIC))
        return m;
    const int axis = sp.dim - 1;
    const int64_t n = sp.n[axis];
    const int64_t row = (int64_t)sp.cells / n;
    const int64_t g = (int64_t)sp.radius * sp.T;
    if (row % 2 != 0 || n < 2) // slab views must start on 16-byte boundaries
        return m;
    const double bytes = (double)sp.cells * sizeof(double);
    m.copy = bytes / kCopyBytesPerSecond;
    m.comp = sp.est_seconds;
    int forced = 0;
    if (const char *env = std::getenv("FFS_HOST_SLABS"))
        forced = std::max(0, std::atoi(env));
    auto model_for = [&](int k, SlabModel *out) {
        const int64_t h = (n + k - 1) / k;
        const int kk = (int)((n + h - 1) / h);
        const bool periodic = sp.boundary == FFS_BOUNDARY_PERIODIC;
        const int64_t rows = periodic ? h + 2 * g : std::min<int64_t>(h + 2 * g, n);
        const int open = periodic ? 0 : (3 << (2 * axis));
        ffs_problem q = slab_problem(sp, rows, open);
        PlanSpec ss;
        std::string why;
        if (build_plan_spec(q, &ss, &why, false) != FFS_OK)
            return false;
        out->count = kk;
        out->a = out->c = (double)h * row * sizeof(double) / kCopyBytesPerSecond;
        out->b = ss.est_seconds + ss.passes * kSlabPassSeconds;
        return true;
    };
    if (forced > 0) {
        SlabModel f = m;
        f.forced = true;
        if (forced > 1 && model_for((int)std::min<int64_t>(forced, n), &f))
            return f;
        return f;
    }
    SlabModel best = m;
    double best_t = m.whole(1);
    for (int k = 2; k <= kMaxSlabs; ++k) {
        const int64_t h = (n + k - 1) / k;
        if (h < 4 * g || (double)h * row * sizeof(double) < (double)kMinSlabBytes)
            break;
        SlabModel c = m;
        if (!model_for(k, &c))
            continue;
        const double t = c.slabs(1);
        if (t < best_t) {
            best_t = t;
            best = c;
        }
    }
    return best;
}

void fill_plan_info(const PlanSpec &sp, ffs_plan_info *info)
{
    memset(info, 0, sizeof(*info));
    info->dim = sp.dim;
    info->radius = sp.radius;
    info->form = sp.form;
    info->tile = sp.tile;
    info->tau = sp.tau;
    info->tau_last = sp.tau_last;
    info->passes = sp.passes;
    info->slices = sp.slices;
    info->host_slabs = slab_model(sp).count;
    info->model_ms = sp.est_seconds * 1e3;
    if (sp.passes > 0) {
        const PassSpec &ps = sp.pass[0];
        info->halo = ps.halo;
        info->useful = ps.useful;
        info->tiles = (sp.dim == 2 && sp.tile == 128) ? ps.nitems : ps.nitems * 2;
        const double n = sp.tile;
        // dense DFT-GEMM count: 2 directions x d axes x n^(d+1) complex MACs x 8 flops, per complex tile
        const double dense = 2.0 * sp.dim * std::pow(n, sp.dim + 1) * 8.0;
        // executed: sum of the radices of the factorisation per axis (8(d) rule n -> n1 + n2):
        // 1D 4096 = 8.8.8.8 -> 32, 2D 64 = 8.8 -> 16, 3D 16 = 4.4 -> 8 (32 = 4.8 -> 12) complex MACs per element
        const double rsum = sp.dim == 1 ? 32.0 : (sp.dim == 2 ? 16.0 : (sp.tile == 32 ? 12.0 : 8.0));
        const double exec = 2.0 * sp.dim * std::pow(n, sp.dim) * rsum * 8.0;
        info->flops_per_pass = dense * (double)ps.nitems;
        info->exec_flops_per_pass = exec * (double)ps.nitems;
        if (sp.form == FFS_FORM_OZAKI_I8 || sp.form == FFS_FORM_BF16X3) {
            const double products = sp.slices * (sp.slices + 1) / 2.0;
            if (sp.dim == 2) // dense DFT-64 GEMMs: 4 stages x (128 x 64 x 128) MACs per slice product
                info->exec_flops_per_pass = 4.0 * 2.0 * 128 * 64 * 128 * products * (double)ps.nitems;
            else // dense DFT-16 GEMMs: 6 stages x (256 lines x 32 x 32) MACs per slice product
                info->exec_flops_per_pass = 6.0 * 2.0 * 256 * 32 * 32 * products * (double)ps.nitems;
        }
        if (sp.form == FFS_FORM_FP64_FFT && sp.dim == 1) {
            // 256 DFT-64 lines per pair (64 rows, 2 x 64 columns, 64 rows) of 8 x (2 x 56 + 7 x 6),
            // two 4096-point twiddle passes (12 per element: table product and multiply), spectrum
            const double line = 8.0 * (2 * 56 + 7 * 6);
            info->exec_flops_per_pass = (256 * line + (2 * 12.0 + 6.0) * 4096) * (double)ps.nitems;
        } else if (sp.form == FFS_FORM_FP64_FFT && sp.dim == 2 && sp.tile == 128) {
            // per FFT-128 line: 8 threads x (DFT-16 of 176 = eight DFT-4 of 16 and eight
            // twiddle products of 6, fifteen w128 twiddles of 6, two DFT-8 of 60); lines per
            // tile: 64 row pairs, 64 columns forward and inverse, u/2 row pairs; plus the
            // spectrum product (6 per point) and the half-spectrum separation (4 per point)
            const double line = 8.0 * (176 + 15 * 6 + 2 * 60);
            info->exec_flops_per_pass = ((64 + 128 + ps.useful / 2.0) * line + 10.0 * 128 * 65) * (double)ps.nitems;
        } else if (sp.form == FFS_FORM_FP64_FFT && sp.dim == 2) {
            // FP64 operations (add = mul = 1, fma = 2) per DFT-64 line: 8 threads x (two DFT-8
            // of 56 + seven twiddle products of 6); lines per pair: 64 rows, 2 x 64 columns and
            // the u wanted rows; plus the spectrum product (6 per element)
            const double line = 8.0 * (2 * 56 + 7 * 6);
            info->exec_flops_per_pass = ((3 * 64 + ps.useful) * line + 6.0 * 64 * 64) * (double)ps.nitems;
        } else if (sp.form == FFS_FORM_FP64_FFT && sp.tile == 32) {
            // per DFT-32 line (4 x 8): eight DFT-4 of 16, 20 twiddle products of 6 (w32^8 is
            // free), four DFT-8 of 60; lines per pair: 1024 each for z, x and y forward and y
            // inverse, 8 u per CTA (32 u) for inverse x, u^2 for inverse z; plus the spectrum
            const double line = 8 * 16 + 20 * 6 + 4 * 60, u = ps.useful;
            info->exec_flops_per_pass = ((4 * 1024 + 32 * u + u * u) * line + 6.0 * 32768) * (double)ps.nitems;
        } else if (sp.form == FFS_FORM_FP64_FFT) {
            // per DFT-16 line: eight DFT-4 of 16 + eight twiddle products of 6 (w16^4 is free);
            // lines per pair: 256 each for x, y, z forward and z inverse, 16 u for inverse y,
            // u^2 for inverse x; plus the spectrum product
            const double line = 8 * 16 + 8 * 6, u = ps.useful;
            info->exec_flops_per_pass = ((4 * 256 + 16 * u + u * u) * line + 6.0 * 4096) * (double)ps.nitems;
        }
        info->hbm_bytes_per_pass = 16.0 * (double)sp.cells;
    }
}

} // namespace ffst

// Describe without allocating (host only).
extern "C" ffs_status ffs_plan_describe(const ffs_problem *problem, ffs_plan_info *info)
{
    if (!problem || !info)
        return ffst::set_error(FFS_ERR_INVALID_ARGUMENT, "ffs_plan_describe: null argument");
    ffst::PlanSpec sp;
    std::string why;
    ffs_status st = ffst::build_plan_spec(*problem, &sp, &why, false);
    if (st != FFS_OK)
        return ffst::set_error(st, why);
    ffst::fill_plan_info(sp, info);
    return FFS_OK;
}
