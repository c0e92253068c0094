// cs3d_dev.cuh -- device-side data structures and helpers shared by the
// kernels of libcs3d.so.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cs3d.h"

namespace cs3d {

constexpr int SLOTS = CS3D_SLOTS;      // node slots per cell (reference padding)
constexpr int NODES = CS3D_NODES;      // real nodes per cell
constexpr int MAXC = CS3D_MAX_CAND;    // contact-candidate cells per cell
constexpr int MAXE = CS3D_MAX_ENTRIES; // contact-candidate nodes per node
constexpr int MAXD = CS3D_MAX_DIS;     // dissipative pairs per node
constexpr int SCAN_TILE = 4096;        // elements per block of the bucket scan
constexpr float DL = 2.9f;             // reference grid spacing, src/GPUbounce.cu:756

// Per-instance constants (uploaded once).
struct InstParams {
    float mass, rr, ra, rs, as, E, stiff1, gint, gext, go, divvol, dt, maxp, minp, growth, thresh;
    float box[3];
    double mass_d;  // mass as a double
    double inv_m;   // 1 / mass, correctly rounded (the integrator's divisions)
    float ra2;      // fl(ra*ra), the reference's float cut-off
    float asE;      // fl(as*E), attraction coefficient
    float rsE;      // fl(rs*E), repulsion coefficient
    float wallk;    // fl(100*E), rigid-box wall stiffness, src/propagate.cu:481
    float rlist;    // neighbour-list radius (ra + skin)
    float skin;     // skin in use (set by the device from the schedule)
    float skin_base;            // the context's skin (CS3D_OPT_SKIN)
    int sk_n;                   // skin schedule by population: ranges in use
    int sk_min[CS3D_SKIN_RANGES];    // lowest cell count of each range, ascending
    float sk_val[CS3D_SKIN_RANGES];  // skin of each range
    int check_sph, angles, rigid, daught_same, div_steps;
    int base, cap;
    int rands;      // Langevin random force on
    float rscale;   // rand_scale_factor
    float rdt;      // sqrtf(dt), the random force's weight in the kicks
    unsigned rseed; // Philox key
    int correct_com;
    int diffE;      // variable stiffness: soft cells lose their pressure from step `phase` on
    float E2;       // stiffness2
    int phase;      // phase_count
    int soften;     // more cells softened at the end of step div_steps + 2
    int soft_n;     // numberOfSofterCells
    float soft_frac;// fractionOfSofterCells (> 0: replaces soft_n)
    int soft_rand;  // RANMAR picks instead of the central cells
    float closeness;// closenessToCenter
    float far_r;    // radius_cutoff of the internal-cells mitotic count (0: off)
};

// Per-instance mutable state (device resident).
struct InstState {
    int n;                 // current cell count
    int step;              // number of the step in progress / last finished
    unsigned err;          // CS3D_ERRBIT_*
    int rebuild;           // list rebuild this step: 0 none, 1 around divisions, 2 whole instance
    float rcur;            // list radius of this step's build
    int mm[2][6];          // grid extents (ordered-int min/max) by step parity
    unsigned disp_step;    // max node displacement of the current step (float bits)
    int div_count;         // divisions in the current step
    int force_rebuild;
    int max_entries, max_cand, max_halo;
    unsigned hbase;        // first bucket of this instance's slice of the node hash
    int hbits;             // log2 of the slice size (0: not rebuilding)
    int built;             // cells whose lists were built (cumulative)
    int rebuilds;
    int rebuilds_div;      // of those, the ones only the rule for dividing instances called for
    float syscm[3];        // the reference's system centre of mass as of its last
                           // calc_sys_CM call, (1, 1, 1) before the first one
    // RANMAR, src/marsaglia.h:50-52
    float u[98];
    float rc, rcd, rcm;
    int i97, j97;
};

struct DivEntry {
    int parent, daughter, inst, pad;
    float n[4];
};

// Static mesh tables in global memory (7 KB, L1/L2 resident).
struct Topo {
    uint32_t *nnpack;   // [192] nn0 | nn1<<8 | nn2<<16 | (sign&0xff)<<24
    float4 *r0;         // [192] equilibrium lengths to nn0..2
    float4 *th0;        // [192] aij, ajk, aik
    double2 *cs0;       // [192*3] (cos, sin) of aij, ajk, aik in FP64
    double *r0i;        // [192*3] 1/R0 in FP64
    uint4 *arm;         // [192] x, y, z: arm-force index n*3 + k for the three neighbours n
    uint8_t *faces;     // [92*7]
};

// Pointers of a context (passed by value to every kernel).
struct Dev {
    int n_inst;
    int cap_total;
    InstParams *prm;
    InstState *st;
    Topo topo;
    float4 *X;          // positions (x, y, z, 0), [cell*192 + node]
    float4 *V;          // velocities (state)
    float4 *Vb;         // velocities after the half kicks (v3), read by neighbours
    float4 *Xe;         // step-end positions kept by the last (fused) S2 of a cs3d_step call
    float4 *FC, *FD;    // forces
    float4 *FR;         // Langevin random force of the last step (zero when off)
    float *stage;       // [6 * cap_total*192] host transfer staging (SoA)
    float4 *CM;         // centre of mass
    float *press, *E, *vol, *area;
    uint8_t *divflag;
    float4 *aabb[2];    // [2*cell] lo, hi  (stale boxes by parity)
    int *cell_inst;
    int *work;          // active cells
    int *work_n;
    int single;         // one instance with base 0: the work table is the identity
    int *cand;          // [cell*MAXC]
    int *ncand;         // [cell]
    float4 *Xb;         // anchors of the displacement test (positions at a build)
    int *dirty;         // [cell] 1: divided last step, 2: within the list radius of such a cell
    // contact candidates of each node: slot << 8 | node, ascending, where
    // slot indexes the cell's candidate list (cand) and node the node in
    // that cell
    uint16_t *ent;      // [(cell*MAXE + k)*192 + node]
    uint8_t *nent;      // [cell*192 + node]
    // the dissipative pairs S1 found this step (slot << 8 | node, in entry
    // order), read by S2: positions do not change in between
    uint16_t *dlist;    // [(cell*MAXD + k)*192 + node]
    uint8_t *ndis;      // [cell*192 + node]
    // node-level spatial hash of the neighbour-list build: cubic bins of
    // edge ~rlist hashed (with the instance) into hsize buckets
    int hsize;          // bucket capacity (>= twice the nodes of the capacity)
    int *hsz;           // buckets in use by the current list build (whole scan tiles, <= hsize)
    int *hcount;        // [hsize + SCAN_TILE] bucket counts, then exclusive starts
    int *hscan;         // [hsize / SCAN_TILE + 1] tile sums of the scan
    float4 *hpos;       // [cap_total*192] positions sorted by bucket, w = (cell << 8 | node) bits
    int *node_rank;     // [cap_total*192] position of the node in its bucket
    DivEntry *divtab;
    int *div_total;
    int4 *events;       // (inst, step, parent, daughter)
    int4 *farlog;       // (inst, step, far cells, 0) of the internal-cells mitotic count
    int *n_far;
    int far_cap;
    uint8_t *pick;      // [cap_total + n_inst] flags of the random soft-cell picks
    int *n_events;
    int ev_cap;
    int *flags;         // [0] any rebuild, [1] any division
    int4 *pairs;        // (cell_a<<8 | node_i, cell_b<<8 | node_j, kind, 0)
    unsigned long long *n_pairs;
    long long pair_cap;
    int record_pairs;
    int halo_stats;     // count distinct candidate nodes per cell at list builds
};

__device__ __forceinline__ int f2o(float f)
{
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// The squared distance of the reference's contact decisions (pair cut-offs,
// box filter) as the reference's own build evaluates dx*dx + dy*dy + dz*dz:
// nvcc's default contraction gives fma(dz, dz, fma(dx, dx, dy*dy)).  Written
// with explicit intrinsics so that no compiler setting can change it.
__device__ __forceinline__ float r2_ref(float dx, float dy, float dz)
{
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// Grid divisions, src/GPUbounce.cu:1332-1334.
__device__ __forceinline__ int grid_div(float mn, float mx)
{
    return (int)__fadd_rn(__fdiv_rn(__fsub_rn(mx, mn), DL), 1.0f);
}

// Node bin along one axis, src/propagate.cu:360-370.
__device__ __forceinline__ int node_bin_axis(float x, float mn, int div)
{
    int s = (int)__fdiv_rn(__fsub_rn(x, mn), DL);
    if (s < 0) s = 0;
    if (s >= div) s = div - 1;
    return s;
}

// makeNNlist insertion range along one axis, src/propagatebound.cu:224-241.
__device__ __forceinline__ void bin_range_axis(float lo, float hi, float attrac, float mn, int div,
                                               int &st, int &en)
{
    st = (int)__fdiv_rn(__fsub_rn(__fsub_rn(lo, attrac), mn), DL);
    if (st < 0) st = 0;
    en = (int)__fdiv_rn(__fsub_rn(__fadd_rn(hi, attrac), mn), DL);
    if (en >= div) en = div - 1;
}

// Bounding-box filter, src/propagate.cu:382-392.  True if the cell is kept.
__device__ __forceinline__ bool aabb_keep(float4 lo, float4 hi, float X, float Y, float Z, float ra2)
{
    float a = __fsub_rn(X, hi.x), b = __fsub_rn(lo.x, X);
    float dx = __fadd_rn(__fmul_rn((float)(a > 0.0f), a), __fmul_rn((float)(b > 0.0f), b));
    a = __fsub_rn(Y, hi.y); b = __fsub_rn(lo.y, Y);
    float dy = __fadd_rn(__fmul_rn((float)(a > 0.0f), a), __fmul_rn((float)(b > 0.0f), b));
    a = __fsub_rn(Z, hi.z); b = __fsub_rn(lo.z, Z);
    float dz = __fadd_rn(__fmul_rn((float)(a > 0.0f), a), __fmul_rn((float)(b > 0.0f), b));
    return !(r2_ref(dx, dy, dz) > ra2);
}

}  // namespace cs3d
