// ref_harness.cu -- drives the reference CellSim3D CUDA kernels, compiled
// unmodified from the reference's own sources (src/propagate.cu,
// src/centermass.cu, src/volume.cu, src/propagatebound.cu,
// src/PressureKernels.cu, src/postscriptinit.cu), through the reference's
// timestep: the launch sequence, launch shapes and host round trips of
// src/GPUbounce.cu:978-1004 (initial forces) and :1055-1338 (one step).
//
// TEST AND BASELINE INFRASTRUCTURE ONLY.  It exists to pin the restatement
// in cellsim3d_b200 against the reference's own arithmetic and to time the
// reference on the same GPU; nothing in the product links or calls it.
//
// What differs from the reference's main(): the initial state (positions,
// velocities, per-cell pressure and stiffness) and the mesh connectivity
// (neighbours, orientation signs, faces) come from an input file instead of
// initialize_C180s / the C180* files.  The equilibrium bond lengths R0 and
// angles theta0 are not taken from the input: they are computed here from
// cell 0 of the input positions with the reference's own float3 helpers
// (inc/VectorFunctions.hpp) and expressions, src/GPUbounce.cu:1890-1908 (R0)
// and :909-935 (theta0).  No trajectory or force files are written, and three
// host-side guards keep the reference's kernels inside the memory they own:
//   * before makeNNlist (host): the grid must fit the per-step clear of the
//     bin counts (cudaMemset of 1 MiB, src/GPUbounce.cu:1329) and the bin
//     lists (32 * bins + cells <= MAX_NN * capacity ints); otherwise the run
//     stops;
//   * after makeNNlist (device): bin counts above the 32 list slots that
//     CalculateConForce/CalculateDisForce read are clamped to 32 (the
//     reference would read past its bin);
//   * before the force kernels (device): where more cells than the 10
//     entries of localNNs (src/propagate.cu:222, :587; the bound check there
//     is against MAX_NN = 1024) pass the bounding-box filter for a node, the
//     bin's count is cut so that no node sees more than 10.
// Clamped or cut counts change the reference's contacts, so such a run is
// flagged (status 1 or 2) and is valid for timing only.
//
// Also driven, as the reference's main does: the CoM correction
// (src/GPUbounce.cu:783-805 at set-up, :1430-1440 every step, with the host's
// calc_sys_CM), the variable-stiffness schedule (PressureUpdate and volumes
// with their stiffness arguments, the growth-end softening of :1340-1429 on
// the host with the reference's ranmar), the internal-cells count of the
// mitotic index (num_cells_far, :2538-2565) and the Langevin force (curand
// MT19937 seeds, DeviceRandInit and CalculateRanForce, :697-730, :1133-1137).
// A growth-end random softening that asks for more distinct cells than
// exist, where the reference loops forever, stops the run (status 6).  The guard kernels
// are asynchronous (no host round trip is added to the step) and their
// device time, measured with events, is excluded from the timing.
//
// Usage: cs3d_ref <in.bin> <out.bin>            (format: oracle/ref.py)
//        cs3d_ref --tables <in.bin> <out.bin>   R0 and theta0 only ("CS3DREFT",
//                                               float32 r0[576], theta0[576]);
//                                               makes no CUDA call
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <cmath>
#include <ctime>
#include <vector>

#include <curand.h>

#include "postscript.h"
#include "marsaglia.h"
#include "RandomVector.h"
#include "VectorFunctions.hpp"

#include "../include/cs3d.h"

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "cs3d_ref: %s: %s (line %d)\n", #call, cudaGetErrorString(e_), __LINE__); \
            exit(2);                                                                   \
        }                                                                              \
    } while (0)

enum {
    ST_OK = 0,
    ST_BIN_OVERFLOW = 1,   // a bin held more than 32 cells (clamped)
    ST_LOCAL_NN = 2,       // more than 10 cells passed the box filter for a node (bin cut)
    ST_NAN = 3,            // NaN position seen
    ST_CAPACITY = 4,       // division past capacity (stopped)
    ST_GRID = 5,           // grid larger than the reference's buffers (stopped)
    ST_SOFT = 6,           // more distinct softer cells requested than exist (stopped)
};

// ---------------------------------------------------------------------------
// guard kernels (not part of the reference's step; timed separately)
// g[0] max bin count, g[1] max cells passing the box filter for a node,
// g[2] NaN seen
// ---------------------------------------------------------------------------
__global__ void guard_bins(int *count, int nbins, int *g)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) {
        const int c = count[b];
        atomicMax(&g[0], c);
        count[b] = c > 32 ? 32 : c;
    }
}

__global__ void guard_cut_init(const int *count, int *cut, int nbins)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) cut[b] = count[b];
}

// The reference's per-node candidate loop (src/propagate.cu:356-404 without
// its stores): where the 11th passing cell would be stored, cut the bin.
__global__ void guard_nodes(int n, const float *X, const float *Y, const float *Z, const float *bb,
                            float Minx, float Miny, float Minz, int Xdiv, int Ydiv, int Zdiv,
                            const int *count, const int *list, int *cut, float DL, float ra, int *g)
{
    const int cell = blockIdx.x, node = threadIdx.x;
    if (cell >= n || node >= 180) return;
    const int gi = cell * 192 + node;
    const float x = X[gi], y = Y[gi], z = Z[gi];
    if (isnan(x) || isnan(y) || isnan(z)) { atomicExch(&g[2], 1); return; }
    int sx = (int)((x - Minx) / DL); if (sx < 0) sx = 0; if (sx >= Xdiv) sx = Xdiv - 1;
    int sy = (int)((y - Miny) / DL); if (sy < 0) sy = 0; if (sy >= Ydiv) sy = Ydiv - 1;
    int sz = (int)((z - Minz) / DL); if (sz < 0) sz = 0; if (sz >= Zdiv) sz = Zdiv - 1;
    const int b = sz * Xdiv * Ydiv + sy * Xdiv + sx;
    int k = 0;
    for (int q = 0; q < count[b]; ++q) {
        const int c = list[32 * b + q];
        if (c == cell) continue;
        float dx = (x - bb[6 * c + 1] > 0.0f) * (x - bb[6 * c + 1]) + (bb[6 * c + 0] - x > 0.0f) * (bb[6 * c + 0] - x);
        float dy = (y - bb[6 * c + 3] > 0.0f) * (y - bb[6 * c + 3]) + (bb[6 * c + 2] - y > 0.0f) * (bb[6 * c + 2] - y);
        float dz = (z - bb[6 * c + 5] > 0.0f) * (z - bb[6 * c + 5]) + (bb[6 * c + 4] - z > 0.0f) * (bb[6 * c + 4] - z);
        if (dx * dx + dy * dy + dz * dz > ra * ra) continue;
        ++k;
        if (k == 11) atomicMin(&cut[b], q);
    }
    atomicMax(&g[1], k);
}

__global__ void guard_cut_apply(int *count, const int *cut, int nbins)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += gridDim.x * blockDim.x) count[b] = cut[b];
}

// ---------------------------------------------------------------------------
struct Input {
    cs3d_params p;
    cs3d_topology t;
    int n, cap, steps, flags, warmup;
    std::vector<float> X, Y, Z, VX, VY, VZ, press, youngs;
};

// The input file must match this harness's compiled layout exactly (sizes written by
// the caller and checked here), and every value the reference kernels index
// with or trap on is validated on the host before any launch: neighbour and
// face indices in range, symmetric neighbour table, positive finite lengths
// and angles, finite state, sane sizes.  A mismatched or corrupt file is
// rejected instead of reaching the GPU.
static bool fail_input(const char *why)
{
    fprintf(stderr, "cs3d_ref: input rejected: %s\n", why);
    return false;
}

// R0 and theta0 from cell 0 of the input, as the reference's set-up computes
// them on the host: R0 = mag(a - b) per bond (src/GPUbounce.cu:1890-1908),
// theta0 = acos of the float dot ratio per vertex angle (:909-935), with the
// reference's float3 helpers (dot, mag, operator-) from inc/VectorFunctions.hpp,
// compiled by the same compiler as the reference's host code.  The input's
// r0 and theta0 are overwritten.
static void ref_tables(Input &in)
{
    const float *X = in.X.data(), *Y = in.Y.data(), *Z = in.Z.data();
    const int *nn = in.t.nn;
    memset(in.t.r0, 0, sizeof in.t.r0);
    memset(in.t.theta0, 0, sizeof in.t.theta0);
    for (int i = 0; i < 180; ++i) {
        const float3 a = make_float3(X[i], Y[i], Z[i]);
        for (int q = 0; q < 3; ++q) {
            const int nb = nn[q * 192 + i];
            const float3 b = make_float3(X[nb], Y[nb], Z[nb]);
            in.t.r0[q * 192 + i] = mag(a - b);
        }
    }
    // theta0 in the angles3 layout {aij, ajk, aik} per node, written as floats
    float *th = in.t.theta0;
    for (int n = 0; n < 180; ++n) {
        const float3 p = make_float3(X[n], Y[n], Z[n]);
        const float3 ni = make_float3(X[nn[n]], Y[nn[n]], Z[nn[n]]) - p;
        const float3 nj = make_float3(X[nn[192 + n]], Y[nn[192 + n]], Z[nn[192 + n]]) - p;
        const float3 nk = make_float3(X[nn[384 + n]], Y[nn[384 + n]], Z[nn[384 + n]]) - p;
        th[3 * n + 0] = acos(dot(ni, nj) / (mag(ni) * mag(nj)));
        th[3 * n + 1] = acos(dot(nj, nk) / (mag(nj) * mag(nk)));
        th[3 * n + 2] = acos(dot(ni, nk) / (mag(ni) * mag(nk)));
    }
}

static bool finite_all(const std::vector<float> &v)
{
    for (float x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

static bool read_input(const char *path, Input &in)
{
    FILE *f = fopen(path, "rb");
    if (!f) return fail_input("cannot open");
    fseek(f, 0, SEEK_END);
    const long fsize = ftell(f);
    fseek(f, 0, SEEK_SET);
    char magic[8];
    int sizes[2] = {0, 0};
    bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "CS3DREF2", 8) == 0;
    if (!ok) { fclose(f); return fail_input("bad magic (stale writer or build)"); }
    ok = fread(sizes, sizeof(int), 2, f) == 2 && sizes[0] == (int)sizeof(cs3d_params) &&
         sizes[1] == (int)sizeof(cs3d_topology);
    if (!ok) { fclose(f); return fail_input("parameter/topology layout differs from this harness (rebuild oracle/_ref)"); }
    ok = fread(&in.p, sizeof in.p, 1, f) == 1 && fread(&in.t, sizeof in.t, 1, f) == 1;
    int hdr[5];
    ok = ok && fread(hdr, sizeof(int), 5, f) == 5;
    if (!ok) { fclose(f); return fail_input("truncated header"); }
    in.n = hdr[0]; in.cap = hdr[1]; in.steps = hdr[2]; in.flags = hdr[3]; in.warmup = hdr[4];
    if (!(in.n >= 1 && in.cap >= in.n && in.cap <= (1 << 22) && in.steps >= 0 && in.steps <= 10000000 &&
          in.warmup >= 0 && in.warmup <= in.steps)) {
        fclose(f);
        return fail_input("sizes out of range");
    }
    const size_t k = (size_t)in.n * 192;
    const long expect = 8 + 8 + (long)sizeof(cs3d_params) + (long)sizeof(cs3d_topology) + 20 +
                        (long)(6 * k + 2 * (size_t)in.n) * 4;
    if (fsize != expect) { fclose(f); return fail_input("file length does not match its header"); }
    std::vector<float> *arr[6] = {&in.X, &in.Y, &in.Z, &in.VX, &in.VY, &in.VZ};
    for (auto *a : arr) { a->resize(k); ok = ok && fread(a->data(), sizeof(float), k, f) == k; }
    in.press.resize(in.n); in.youngs.resize(in.n);
    ok = ok && fread(in.press.data(), sizeof(float), in.n, f) == (size_t)in.n;
    ok = ok && fread(in.youngs.data(), sizeof(float), in.n, f) == (size_t)in.n;
    fclose(f);
    if (!ok) return fail_input("truncated arrays");
    for (auto *a : arr)
        if (!finite_all(*a)) return fail_input("non-finite position or velocity");
    if (!finite_all(in.press) || !finite_all(in.youngs)) return fail_input("non-finite pressure or stiffness");
    const cs3d_params &p = in.p;
    if (!(p.particle_mass > 0 && p.time_interval > 0 && p.time_interval < 1 && p.attraction_range > 0 &&
          p.attraction_range < 10 && p.repulsion_range >= 0 && std::isfinite(p.youngs_mod) &&
          std::isfinite(p.stiffness1) && std::isfinite(p.max_pressure) && std::isfinite(p.min_pressure) &&
          std::isfinite(p.growth_rate) && std::isfinite(p.division_vol)))
        return fail_input("parameters out of range");
    if (!(std::isfinite(p.rand_scale_factor) && std::isfinite(p.stiffness2) && p.number_of_softer_cells >= 0 &&
          std::isfinite(p.fraction_of_softer_cells) && std::isfinite(p.closeness_to_center) &&
          std::isfinite(p.count_internal_radius)))
        return fail_input("schedule parameters out of range");
    for (int q = 0; q < 3; ++q)
        for (int i = 0; i < 180; ++i) {
            const int nb = in.t.nn[q * 192 + i];
            if (nb < 0 || nb >= 180) return fail_input("neighbour index out of range");
            bool back = false;
            for (int m = 0; m < 3; ++m) back = back || in.t.nn[m * 192 + nb] == i;
            if (!back) return fail_input("neighbour table not symmetric");
        }
    for (int i = 0; i < 180; ++i)
        if (in.t.sign[i] != 1 && in.t.sign[i] != -1) return fail_input("bad orientation sign");
    for (int fc = 0; fc < 92; ++fc)
        for (int m = 0; m < (fc < 12 ? 5 : 6); ++m) {
            const int v = in.t.faces[fc * 7 + m];
            if (v < 0 || v >= 180) return fail_input("face index out of range");
        }
    // the reference's own equilibrium tables from cell 0 of the input
    ref_tables(in);
    for (int q = 0; q < 3; ++q)
        for (int i = 0; i < 180; ++i) {
            const float r0 = in.t.r0[q * 192 + i];
            if (!(r0 > 0 && r0 < 10)) return fail_input("bond length out of range");
        }
    for (int i = 0; i < 3 * 180; ++i)
        if (!(in.t.theta0[i] > 0 && in.t.theta0[i] < 3.1416f)) return fail_input("angle out of range");
    return true;
}

template <typename T> static T *dev(size_t n)
{
    T *p = nullptr;
    CK(cudaMalloc(&p, n * sizeof(T) + 256));
    CK(cudaMemset(p, 0, n * sizeof(T) + 256));
    return p;
}

int main(int argc, char **argv)
{
    const bool tables_only = argc == 4 && strcmp(argv[1], "--tables") == 0;
    if (argc != 3 && !tables_only) {
        fprintf(stderr, "usage: %s [--tables] in.bin out.bin\n", argv[0]);
        return 1;
    }
    if (tables_only) { ++argv; }
    Input in;
    if (!read_input(argv[1], in)) { fprintf(stderr, "cs3d_ref: bad input %s\n", argv[1]); return 1; }
    if (tables_only) {
        // R0 and theta0 only: no CUDA call, so this runs on a host without a GPU
        FILE *ft = fopen(argv[2], "wb");
        if (!ft) { fprintf(stderr, "cs3d_ref: cannot write %s\n", argv[2]); return 1; }
        fwrite("CS3DREFT", 1, 8, ft);
        fwrite(in.t.r0, sizeof(float), 576, ft);
        fwrite(in.t.theta0, sizeof(float), 576, ft);
        fclose(ft);
        return 0;
    }
    const cs3d_params &p = in.p;
    const int cap = in.cap;
    const size_t NS = (size_t)192 * cap;
    const int threadsperblock = 192;
    const float DL = 2.9f;

    // device buffers, sizes of src/GPUbounce.cu:365-415
    float *d_X = dev<float>(NS), *d_Y = dev<float>(NS), *d_Z = dev<float>(NS);
    float *d_XP = dev<float>(NS), *d_YP = dev<float>(NS), *d_ZP = dev<float>(NS);
    float *d_XM = dev<float>(NS), *d_YM = dev<float>(NS), *d_ZM = dev<float>(NS);
    float *d_vx = dev<float>(NS), *d_vy = dev<float>(NS), *d_vz = dev<float>(NS);
    R3Nptrs fCon{dev<float>(NS), dev<float>(NS), dev<float>(NS)};
    R3Nptrs fDis{dev<float>(NS), dev<float>(NS), dev<float>(NS)};
    R3Nptrs fRan{dev<float>(NS), dev<float>(NS), dev<float>(NS)};
    R3Nptrs contact{dev<float>(NS), dev<float>(NS), dev<float>(NS)};
    float *d_CMx = dev<float>(cap), *d_CMy = dev<float>(cap), *d_CMz = dev<float>(cap);
    float *d_bb = dev<float>((size_t)6 * cap);
    float *d_Minx = dev<float>(1024), *d_Maxx = dev<float>(1024), *d_Miny = dev<float>(1024);
    float *d_Maxy = dev<float>(1024), *d_Minz = dev<float>(1024), *d_Maxz = dev<float>(1024);
    int *d_NoofNNlist = dev<int>(1024 * 1024);
    int *d_NNlist = dev<int>((size_t)MAX_NN * cap);
    float *d_press = dev<float>(cap), *d_E = dev<float>(cap), *d_vol = dev<float>(cap), *d_area = dev<float>(cap);
    char *d_cell_div = dev<char>(cap);
    int *d_nn = dev<int>(3 * 192), *d_sign = dev<int>(180), *d_faces = dev<int>(92 * 7);
    float *d_R0 = dev<float>(3 * 192);
    angles3 *d_theta0 = dev<angles3>(192);
    float *d_time = dev<float>(1), *d_boxMin = dev<float>(3), *d_ran2 = dev<float>(3);
    int *d_reset = dev<int>(2 * (size_t)cap + 2);
    int *d_gmax = dev<int>(4);
    curandState *d_rng = nullptr;
    if (p.add_rands) {
        // src/GPUbounce.cu:697-730
        d_rng = dev<curandState>(NS);
        // MT19937 output lengths are whole multiples of 2048 values; the
        // first NS seed the node states
        const size_t NSR = (NS + 2047) / 2048 * 2048;
        unsigned *d_seeds = dev<unsigned>(NSR);
        curandGenerator_t gen;
        if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_MT19937) != CURAND_STATUS_SUCCESS ||
            curandSetPseudoRandomGeneratorSeed(gen, p.rand_seed > 0 ? (unsigned long long)p.rand_seed
                                                                    : (unsigned long long)time(nullptr)) !=
                CURAND_STATUS_SUCCESS ||
            curandGenerate(gen, d_seeds, NSR) != CURAND_STATUS_SUCCESS) {
            fprintf(stderr, "cs3d_ref: curand set-up failed\n");
            return 2;
        }
        DeviceRandInit<<<(unsigned)(NS / 256 + 1), 256>>>(d_rng, d_seeds, NS);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        curandDestroyGenerator(gen);
        CK(cudaFree(d_seeds));
    }
    // the reference's host system centre (globals, src/GPUbounce.cu:240) and
    // its calc_sys_CM / getRmax2 (:2504-2536) on a host copy of the centres
    float sysCM[3] = {1.0f, 1.0f, 1.0f};
    std::vector<float> hcx(cap), hcy(cap), hcz(cap);
    auto fetch_cm = [&](int n) {
        CK(cudaMemcpy(hcx.data(), d_CMx, n * sizeof(float), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hcy.data(), d_CMy, n * sizeof(float), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hcz.data(), d_CMz, n * sizeof(float), cudaMemcpyDeviceToHost));
    };
    auto calc_sys_cm = [&](int n) {
        float sx = 0, sy = 0, sz = 0;
        for (int c = 0; c < n; ++c) { sx += hcx[c]; sy += hcy[c]; sz += hcz[c]; }
        sysCM[0] = sx / n; sysCM[1] = sy / n; sysCM[2] = sz / n;
    };
    auto dist2 = [&](int c) {
        float dx = hcx[c] - sysCM[0], dy = hcy[c] - sysCM[1], dz = hcz[c] - sysCM[2];
        return dx * dx + dy * dy + dz * dz;
    };
    auto get_rmax2 = [&](int n) {
        float r2 = 0;
        for (int c = 0; c < n; ++c) r2 = std::max(r2, dist2(c));
        return r2;
    };
    std::vector<int> far_log;

    // initial state and tables
    const size_t k0 = (size_t)192 * in.n;
    CK(cudaMemcpy(d_X, in.X.data(), k0 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_Y, in.Y.data(), k0 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_Z, in.Z.data(), k0 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_XP, d_X, k0 * 4, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(d_YP, d_Y, k0 * 4, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(d_ZP, d_Z, k0 * 4, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(d_XM, d_X, k0 * 4, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(d_YM, d_Y, k0 * 4, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(d_ZM, d_Z, k0 * 4, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(d_vx, in.VX.data(), k0 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_vy, in.VY.data(), k0 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_vz, in.VZ.data(), k0 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_press, in.press.data(), in.n * 4, cudaMemcpyHostToDevice));
    std::vector<float> youngs(cap, p.stiffness1);
    for (int c = 0; c < in.n; ++c) youngs[c] = in.youngs[c];
    CK(cudaMemcpy(d_E, youngs.data(), cap * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_nn, in.t.nn, sizeof in.t.nn, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_sign, in.t.sign, sizeof in.t.sign, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_faces, in.t.faces, sizeof in.t.faces, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_R0, in.t.r0, sizeof in.t.r0, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_theta0, in.t.theta0, sizeof in.t.theta0, cudaMemcpyHostToDevice));
    const float delta_t = p.time_interval;
    CK(cudaMemcpy(d_time, &delta_t, 4, cudaMemcpyHostToDevice));
    rmarin(p.rng_ij, p.rng_kl);

    int N = in.n;
    const float ra = p.attraction_range, rr = p.repulsion_range;
    const float3 boxMax = make_float3(p.box_len[0], p.box_len[1], p.box_len[2]);
    const float r_CM_o = pow((3.0 / 4.0) * (1 / 3.14159) * p.division_vol * 2.0, 1.0 / 3);
    const float E = p.youngs_mod;
    int status = ST_OK;
    float Minx[6];
    int Xdiv = 1, Ydiv = 1, Zdiv = 1;
    long long nbins = 1;
    std::vector<int> events;
    int *d_cut = dev<int>(1024 * 1024);

    // guard device time: one event pair per guard launch group
    std::vector<cudaEvent_t> gev;
    auto gmark = [&]() {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        CK(cudaEventRecord(e));
        gev.push_back(e);
    };

    // grid of src/GPUbounce.cu:1312-1337, with the guards around makeNNlist
    auto grid = [&]() -> int {
        bounding_boxes<<<N, 32>>>(N, d_X, d_Y, d_Z, d_bb, d_CMx, d_CMy, d_CMz);
        const int rb = (N - 1) / 1024 + 1;
        minmaxpre<<<rb, 1024>>>(N, d_bb, d_Minx, d_Maxx, d_Miny, d_Maxy, d_Minz, d_Maxz);
        minmaxpost<<<1, 1024>>>(rb, d_Minx, d_Maxx, d_Miny, d_Maxy, d_Minz, d_Maxz);
        CK(cudaMemset(d_NoofNNlist, 0, 1024 * 1024));
        CK(cudaMemcpy(Minx, d_Minx, 6 * sizeof(float), cudaMemcpyDeviceToHost));
        Xdiv = (int)((Minx[1] - Minx[0]) / DL + 1);
        Ydiv = (int)((Minx[3] - Minx[2]) / DL + 1);
        Zdiv = (int)((Minx[5] - Minx[4]) / DL + 1);
        nbins = (long long)Xdiv * Ydiv * Zdiv;
        if (Xdiv < 1 || Ydiv < 1 || Zdiv < 1 || nbins > 1024 * 1024 / 4 || 32 * nbins + N > (long long)MAX_NN * cap)
            return ST_GRID;
        makeNNlist<<<N / 512 + 1, 512>>>(N, d_bb, Minx[0], Minx[2], Minx[4], ra, Xdiv, Ydiv, Zdiv, d_NoofNNlist,
                                          d_NNlist, DL);
        gmark();
        guard_bins<<<256, 256>>>(d_NoofNNlist, (int)nbins, d_gmax);
        gmark();
        return ST_OK;
    };
    // cut bins so that no node stores more than 10 cells (before the forces)
    auto guard_forces = [&]() {
        gmark();
        guard_cut_init<<<256, 256>>>(d_NoofNNlist, d_cut, (int)nbins);
        guard_nodes<<<N, 192>>>(N, d_X, d_Y, d_Z, d_bb, Minx[0], Minx[2], Minx[4], Xdiv, Ydiv, Zdiv, d_NoofNNlist,
                                d_NNlist, d_cut, DL, ra, d_gmax);
        guard_cut_apply<<<256, 256>>>(d_NoofNNlist, d_cut, (int)nbins);
        gmark();
    };
    auto con_force = [&]() {
        CalculateConForce<<<N, threadsperblock>>>(N, d_nn, d_sign, d_X, d_Y, d_Z, d_CMx, d_CMy, d_CMz, d_R0, d_press, d_E,
                                                  p.stiffness1, p.internal_damping, d_time, d_bb, p.attraction_strength,
                                                  ra, p.repulsion_strength, rr, p.viscotic_damping, p.particle_mass,
                                                  Minx[0], Minx[2], Minx[4], Xdiv, Ydiv, Zdiv, d_NoofNNlist, d_NNlist, DL,
                                                  p.gamma_visc, 0.0f, 0.0f, p.thresh_dist, false, d_vx, d_vy, d_vz,
                                                  p.use_rigid_box != 0, 0.0f, d_boxMin, E, p.constrain_angles != 0,
                                                  d_theta0, fCon, r_CM_o, boxMax, contact, d_vol, p.division_vol);
    };
    auto dis_force = [&]() {
        CalculateDisForce<<<N, threadsperblock>>>(N, d_nn, d_sign, d_X, d_Y, d_Z, p.internal_damping, d_bb, ra,
                                                  p.viscotic_damping, Minx[0], Minx[2], Minx[4], Xdiv, Ydiv, Zdiv,
                                                  d_NoofNNlist, d_NNlist, DL, p.gamma_visc, d_vx, d_vy, d_vz, fDis);
    };

    // initialisation, src/GPUbounce.cu:739-763 and :978-1004
    CenterOfMass<<<N, 256>>>(N, d_X, d_Y, d_Z, d_CMx, d_CMy, d_CMz);
    status = grid();
    // flags bit 2: the reference's own grid after this first makeNNlist (bin
    // counts, bin lists, bounding boxes, extents), read back as it left them
    std::vector<int> g_counts, g_list;
    std::vector<float> g_bb;
    float g_minx[6] = {0, 0, 0, 0, 0, 0};
    int g_div[4] = {0, 0, 0, 0};
    if ((in.flags & 4) && status == ST_OK) {
        CK(cudaDeviceSynchronize());
        g_counts.resize(nbins);
        g_list.resize((size_t)32 * nbins);
        g_bb.resize((size_t)6 * N);
        CK(cudaMemcpy(g_counts.data(), d_NoofNNlist, sizeof(int) * nbins, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(g_list.data(), d_NNlist, sizeof(int) * 32 * nbins, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(g_bb.data(), d_bb, sizeof(float) * 6 * N, cudaMemcpyDeviceToHost));
        memcpy(g_minx, Minx, sizeof g_minx);
        g_div[0] = Xdiv; g_div[1] = Ydiv; g_div[2] = Zdiv; g_div[3] = (int)nbins;
    }
    if (p.correct_com) {
        // src/GPUbounce.cu:783-805
        CenterOfMass<<<N, 256>>>(N, d_X, d_Y, d_Z, d_CMx, d_CMy, d_CMz);
        fetch_cm(N);
        calc_sys_cm(N);
        const long np = (long)N * 192;
        CorrectCoMMotion<<<(unsigned)(np / 1024 + 1), 1024>>>(d_X, d_Y, d_Z, sysCM[0], sysCM[1], sysCM[2], np);
        CorrectCoMMotion<<<(unsigned)(np / 1024 + 1), 1024>>>(d_XP, d_YP, d_ZP, sysCM[0], sysCM[1], sysCM[2], np);
        CorrectCoMMotion<<<(unsigned)(np / 1024 + 1), 1024>>>(d_XM, d_YM, d_ZM, sysCM[0], sysCM[1], sysCM[2], np);
        CK(cudaGetLastError());
    }
    const int n_init = N;
    std::vector<float> first_forces;
    if (status == ST_OK) {
        guard_forces();
        con_force();
        dis_force();
        CK(cudaGetLastError());
        if (in.flags & 1) {
            first_forces.resize((size_t)6 * n_init * 192);
            for (int q = 0; q < 6; ++q) {
                const float *s = q < 3 ? (&fCon.x)[q] : (&fDis.x)[q - 3];
                CK(cudaMemcpy(first_forces.data() + (size_t)q * n_init * 192, s, (size_t)n_init * 192 * 4,
                              cudaMemcpyDeviceToHost));
            }
        }
    }
    CK(cudaDeviceSynchronize());
    for (cudaEvent_t e : gev) cudaEventDestroy(e);
    gev.clear();

    // the timestep, src/GPUbounce.cu:1055-1338
    const int Time_steps = p.div_time_steps;
    const float rGrowth = p.growth_rate;
    std::vector<char> cell_div(cap);
    std::vector<int> reset(2 * (size_t)cap + 2);
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    int steps_done = 0;
    if (in.warmup == 0) CK(cudaEventRecord(t0));
    // flags bit 1: colony mode, device time at the first step with N >= 10, 100,
    // 1000 and 4096 cells (the population decades), ending at 4096
    const int marks_at[4] = {10, 100, 1000, 4096};
    int next_mark = 0;
    std::vector<int> marks;
    std::vector<float> mark_ms;
    for (int step = 1; step <= in.steps && status == ST_OK; ++step) {
        const long numNodes = (long)N * 192;
        Integrate<<<N, threadsperblock>>>(d_XP, d_YP, d_ZP, d_X, d_Y, d_Z, d_XM, d_YM, d_ZM, d_vx, d_vy, d_vz, d_time,
                                          p.particle_mass, fCon, fDis, fRan, N, p.add_rands != 0, d_rng,
                                          p.rand_scale_factor);
        ForwardTime<<<N, threadsperblock>>>(d_XP, d_YP, d_ZP, d_X, d_Y, d_Z, d_XM, d_YM, d_ZM, N);
        PressureUpdate<<<N / 1024 + 1, 1024>>>(d_press, p.min_pressure, p.max_pressure, rGrowth, N,
                                               p.use_different_stiffnesses != 0, p.stiffness1, d_E, step,
                                               p.phase_count);
        guard_forces();
        con_force();
        dis_force();
        if (p.add_rands) CalculateRanForce<<<N, threadsperblock>>>(N, d_rng, p.rand_scale_factor, fRan);
        VelocityUpdateA<<<N, threadsperblock>>>(d_vx, d_vy, d_vz, fCon, fRan, delta_t, numNodes, p.particle_mass);
        VelocityUpdateB<<<N, threadsperblock>>>(d_vx, d_vy, d_vz, fDis, delta_t, numNodes, p.particle_mass);
        dis_force();
        CenterOfMass<<<N, 256>>>(N, d_X, d_Y, d_Z, d_CMx, d_CMy, d_CMz);
        if (step <= Time_steps && rGrowth > 0) {
            volumes<<<N, 192>>>(N, d_faces, d_X, d_Y, d_Z, d_CMx, d_CMy, d_CMz, d_vol, d_cell_div, p.division_vol,
                                p.check_sphericity != 0, d_area, p.phase_count, step, p.stiffness1,
                                p.use_different_stiffnesses != 0, d_E, false);
            // count_and_get_div, src/GPUbounce.cu:2489-2500
            CK(cudaMemcpy(cell_div.data(), d_cell_div, N, cudaMemcpyDeviceToHost));
            std::vector<int> divs;
            for (int c = 0; c < N; ++c)
                if (cell_div[c] == 1) { cell_div[c] = 0; divs.push_back(c); }
            CK(cudaMemcpy(d_cell_div, cell_div.data(), N, cudaMemcpyHostToDevice));
            const int nd = (int)divs.size();
            for (int q = 0; q < nd; ++q) {
                if (N + 1 > cap) { status = ST_CAPACITY; break; }
                float norm[3] = {0.f, 1.f, 0.f};
                GetRandomVector(norm);
                CK(cudaMemcpy(d_ran2, norm, 3 * sizeof(float), cudaMemcpyHostToDevice));
                cell_division<<<1, 256>>>(divs[q], d_XP, d_YP, d_ZP, d_X, d_Y, d_Z, d_XM, d_YM, d_ZM, d_CMx, d_CMy,
                                          d_CMz, d_vx, d_vy, d_vz, N, d_ran2, rr);
                reset[q] = divs[q];
                reset[q + nd] = N;
                youngs[N] = p.daught_same_stiffness ? youngs[divs[q]] : p.stiffness1;
                events.push_back(step); events.push_back(divs[q]); events.push_back(N);
                ++N;
            }
            if (status != ST_OK) break;
            if (nd > 0) {
                CK(cudaMemcpy(d_reset, reset.data(), 2 * nd * sizeof(int), cudaMemcpyHostToDevice));
                PressureReset<<<(2 * nd) / 512 + 1, 512>>>(d_reset, d_press, p.min_pressure, 2 * nd);
                CK(cudaMemcpy(d_E, youngs.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
            }
            // num_cells_far, src/GPUbounce.cu:1288-1290, :2538-2565
            if (p.count_internal_radius > 0 && nd > 0 && N >= 50) {
                fetch_cm(N);
                calc_sys_cm(N);
                const float rf = p.count_internal_radius;
                const float thr = rf * rf * get_rmax2(N);
                int far = 0;
                for (int c = N - nd; c < N; ++c)
                    if (dist2(c) > thr) ++far;
                if (far) { far_log.push_back(step); far_log.push_back(far); }
            }
        }
        status = grid();
        CK(cudaGetLastError());
        if (status == ST_OK && p.use_different_stiffnesses && p.soften_after_growth && step == Time_steps + 2) {
            // src/GPUbounce.cu:1340-1429, at the end of the first step after Time_steps + 1
            int count = p.number_of_softer_cells;
            if (p.fraction_of_softer_cells > 0) count = roundf(p.fraction_of_softer_cells * N);
            if (p.choose_random_cell_indices) {
                if (count > N + 1) {
                    status = ST_SOFT;
                } else {
                    std::vector<int> chosen;
                    while ((int)chosen.size() < count) {
                        float rnd[1];
                        ranmar(rnd, 1);
                        const int ind = roundf(rnd[0] * N);
                        bool seen = false;
                        for (int q : chosen) seen = seen || q == ind;
                        if (!seen) chosen.push_back(ind);
                    }
                    // index N names no cell (a division overwrites it before any use)
                    for (int q : chosen)
                        if (q < N) youngs[q] = p.stiffness2;
                }
            } else {
                fetch_cm(N);
                const float rmax2 = get_rmax2(N);   // before calc_sys_CM, as the reference
                calc_sys_cm(N);
                const float f = 1 - p.closeness_to_center;
                int got = 0;
                for (int c = 0; got < count && c < N; ++c)
                    if (dist2(c) <= f * f * rmax2) { youngs[c] = p.stiffness2; ++got; }
            }
            CK(cudaMemcpy(d_E, youngs.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
        }
        if (status == ST_OK && p.correct_com) {
            // src/GPUbounce.cu:1430-1440
            fetch_cm(N);
            calc_sys_cm(N);
            const long np = (long)N * 192;
            CorrectCoMMotion<<<(unsigned)(np / 1024 + 1), 1024>>>(d_X, d_Y, d_Z, sysCM[0], sysCM[1], sysCM[2], np);
            CK(cudaGetLastError());
        }
        if (status == ST_OK) steps_done = step;
        if ((in.flags & 2) && status == ST_OK && next_mark < 4 && N >= marks_at[next_mark]) {
            // the population reached the next decade: device time so far, guard
            // kernels excluded; the run ends at the last one
            cudaEvent_t em;
            CK(cudaEventCreate(&em));
            CK(cudaEventRecord(em));
            CK(cudaEventSynchronize(em));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, t0, em));
            CK(cudaEventDestroy(em));
            double g = 0.0;
            for (size_t q = 0; q + 1 < gev.size(); q += 2) {
                float gm = 0.f;
                cudaEventElapsedTime(&gm, gev[q], gev[q + 1]);
                g += gm;
            }
            marks.push_back(step);
            marks.push_back(N);
            mark_ms.push_back((float)(ms - g));
            ++next_mark;
            if (next_mark == 4) break;
        }
        if (step == in.warmup) {
            // timed region starts after the warm-up steps: drop their guard events
            CK(cudaDeviceSynchronize());
            for (cudaEvent_t e : gev) cudaEventDestroy(e);
            gev.clear();
            CK(cudaEventRecord(t0));
        }
    }
    CK(cudaEventRecord(t1));
    CK(cudaEventSynchronize(t1));
    float total_ms = 0.f;
    cudaEventElapsedTime(&total_ms, t0, t1);
    double guard_ms = 0.0;
    for (size_t q = 0; q + 1 < gev.size(); q += 2) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, gev[q], gev[q + 1]);
        guard_ms += ms;
    }
    int h[3];
    CK(cudaMemcpy(h, d_gmax, 3 * sizeof(int), cudaMemcpyDeviceToHost));
    const int max_bin = h[0], max_nn = h[1];
    if (status == ST_OK && h[2]) status = ST_NAN;
    if (status == ST_OK && max_nn > 10) status = ST_LOCAL_NN;
    if (status == ST_OK && max_bin > 32) status = ST_BIN_OVERFLOW;

    // output
    FILE *fo = fopen(argv[2], "wb");
    if (!fo) { fprintf(stderr, "cs3d_ref: cannot write %s\n", argv[2]); return 1; }
    auto dump3 = [&](const float *a, const float *b, const float *c, int n) {
        std::vector<float> hb((size_t)n * 192);
        for (const float *s : {a, b, c}) {
            CK(cudaMemcpy(hb.data(), s, hb.size() * 4, cudaMemcpyDeviceToHost));
            fwrite(hb.data(), 4, hb.size(), fo);
        }
    };
    fwrite("CS3DREFO", 1, 8, fo);
    const int hdr[6] = {status, steps_done, N, (int)(events.size() / 3), max_bin, max_nn};
    fwrite(hdr, sizeof(int), 6, fo);
    const float tm[2] = {total_ms, (float)guard_ms};
    fwrite(tm, sizeof(float), 2, fo);
    fwrite(events.data(), sizeof(int), events.size(), fo);
    dump3(d_X, d_Y, d_Z, N);
    dump3(d_vx, d_vy, d_vz, N);
    dump3(fCon.x, fCon.y, fCon.z, N);
    dump3(fDis.x, fDis.y, fDis.z, N);
    std::vector<float> hp(N);
    CK(cudaMemcpy(hp.data(), d_press, N * 4, cudaMemcpyDeviceToHost));
    fwrite(hp.data(), 4, N, fo);
    CK(cudaMemcpy(hp.data(), d_E, N * 4, cudaMemcpyDeviceToHost));
    fwrite(hp.data(), 4, N, fo);
    std::vector<float> hcm(3 * (size_t)N);
    CK(cudaMemcpy(hcm.data(), d_CMx, N * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hcm.data() + N, d_CMy, N * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hcm.data() + 2 * N, d_CMz, N * 4, cudaMemcpyDeviceToHost));
    fwrite(hcm.data(), 4, hcm.size(), fo);
    const int nf = (int)first_forces.size();
    fwrite(&n_init, sizeof(int), 1, fo);
    fwrite(&nf, sizeof(int), 1, fo);
    if (nf) fwrite(first_forces.data(), 4, first_forces.size(), fo);
    dump3(fRan.x, fRan.y, fRan.z, N);
    const int nfar = (int)(far_log.size() / 2);
    fwrite(&nfar, sizeof(int), 1, fo);
    if (nfar) fwrite(far_log.data(), sizeof(int), far_log.size(), fo);
    const int nmark = (int)mark_ms.size();
    fwrite(&nmark, sizeof(int), 1, fo);
    for (int q = 0; q < nmark; ++q) {
        fwrite(&marks[2 * q], sizeof(int), 2, fo);
        fwrite(&mark_ms[q], sizeof(float), 1, fo);
    }
    const int ngrid = (int)g_bb.size() / 6;
    fwrite(&ngrid, sizeof(int), 1, fo);
    if (ngrid) {
        fwrite(g_minx, sizeof(float), 6, fo);
        fwrite(g_div, sizeof(int), 4, fo);
        fwrite(g_counts.data(), sizeof(int), g_counts.size(), fo);
        fwrite(g_list.data(), sizeof(int), g_list.size(), fo);
        fwrite(g_bb.data(), sizeof(float), g_bb.size(), fo);
    }
    fclose(fo);
    for (cudaEvent_t e : gev) cudaEventDestroy(e);
    return 0;
}
