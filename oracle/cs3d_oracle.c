/*
 * cs3d_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of CellSim3D's per-timestep loop, used as the parity oracle
 * for the CUDA path in cellsim3d_b200.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load this library; the product never
 * links or calls it.
 *
 * Arithmetic contract (the oracle is the FP64 "truth" with FP32 decisions):
 *   - State (positions, velocities, pressures, stiffness, CoM, bounding boxes)
 *     is stored in float, exactly as the reference keeps it.
 *   - Force values, CoM, volume, area and division geometry are evaluated in
 *     double from the float state.
 *   - Every discrete decision that the reference makes in float (contact-pair
 *     cut-offs, bounding-box filter, bin indices, wall gaps, grid extents) is
 *     evaluated in float with the reference's expression order, as the
 *     reference's own nvcc build evaluates it: no contraction of its own
 *     (built with -ffp-contract=off) except the squared distances of the
 *     contact decisions, which that build fuses into FMAs (r2_ref below), so
 *     the pair sets are exact.
 *   - RANMAR and the Marsaglia sphere point are float, bit-exact.
 *
 * Reference files cited as path:line within SoftSimu/CellSim3D.
 * Parity pinning: RANMAR against the known-answer values in
 * src/marsaglia.h:66-72; forces, pairs and division against the reference
 * CUDA kernels built from their own sources (oracle/_ref), see tests/.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define ORC_SLOTS 192       /* nodes per cell slot, src/GPUbounce.cu:365 */
#define ORC_NODES 180
#define ORC_DL 2.9f         /* grid spacing, src/GPUbounce.cu:756 */
#define ORC_MAX_EVENTS (1 << 20)

/* error bits reported by the oracle (same meaning as the CUDA path's) */
#define ORC_ERR_NAN            0x1u
#define ORC_ERR_CAPACITY       0x2u
#define ORC_ERR_BIN_OVERFLOW   0x4u   /* a reference bin would hold > 32 cells */
#define ORC_ERR_LOCALNN        0x8u   /* a node would accept > 10 cells */
#define ORC_ERR_MEMSET_BUG     0x10u  /* > 262144 bins: reference leaves stale counts */
#define ORC_ERR_NONFINITE_VOL  0x20u
#define ORC_ERR_SOFT_CELLS     0x40u  /* more softer cells than indices: the reference loops forever */

typedef struct {
    float mass;               /* core.particle_mass */
    float rep_range;          /* core.repulsion_range */
    float att_range;          /* core.attraction_range */
    float rep_strength;       /* core.repulsion_strength */
    float att_strength;       /* core.attraction_strength */
    float youngs_mod;         /* core.Youngs_mod */
    float stiffness1;         /* core.stiffFactor1 * Youngs_mod */
    float gamma_int;          /* core.internal_damping */
    float gamma_ext;          /* core.viscotic_damping */
    float gamma_o;            /* core.gamma_visc */
    float div_vol;            /* core.division_Vol */
    float dt;                 /* core.time_interval */
    float max_p, min_p;       /* core.maxPressure, core.minPressure */
    float growth_rate;        /* core.growth_rate */
    float thresh_dist;        /* walls.threshDist */
    float box[3];             /* boxParams.box_len_{x,y,z} */
    int check_sphericity;
    int constrain_angles;
    int use_rigid_box;
    int daught_same_stiffness;
    int div_time_steps;       /* core.div_time_steps */
    int pad_;
    int add_rands;            /* rand_params.add_rands */
    float rand_scale;         /* rand_params.rand_scale_factor */
    unsigned rand_seed;       /* Philox key (see orc_random_force) */
    int correct_com;          /* core.correct_com */
    int diff_stiff;           /* stiffnessParams.useDifferentStiffnesses */
    float stiffness2;         /* softStiffFactor * Youngs_mod */
    int phase_count;          /* core.phase_count */
    int soften_after_growth;  /* !stiffnessParams.duringGrowth */
    int soft_n;               /* numberOfSofterCells */
    float soft_frac;          /* fractionOfSofterCells */
    int soft_rand;            /* chooseRandomCellIndices */
    float closeness;          /* closenessToCenter */
    float far_r;              /* radius_cutoff when count_only_internal_cells (else 0) */
} orc_params;

typedef struct {
    int nn[3 * ORC_SLOTS];      /* 0-based neighbour ids, [k*192 + node] */
    int sign[ORC_NODES];
    float r0[3 * ORC_SLOTS];    /* [k*192 + node] */
    float theta0[3 * ORC_SLOTS];/* [node*3 + {aij, ajk, aik}] */
    int faces[92 * 7];          /* C180_56 layout, src/GPUbounce.cu:1861-1886 */
} orc_topo;

typedef struct {
    float u[98];
    float c, cd, cm;
    int i97, j97;
    int ok;
} orc_ranmar;

typedef struct orc_sys {
    int cap, n;
    orc_params P;
    orc_topo T;
    float *X, *Y, *Z, *VX, *VY, *VZ;
    double *FC, *FD;           /* [3][cap*192] */
    float *FR;                 /* [3][cap*192] random force of the last step */
    float *CM;                 /* [3][cap] */
    float *press, *E, *vol, *area;
    unsigned char *div_flag;
    float *aabb;               /* [cap*6]: minx maxx miny maxy minz maxz */
    float minmax[6];
    int xdiv, ydiv, zdiv;
    /* reference neighbour bins (unbounded CSR; overflow past 32 is flagged) */
    int nbins;
    int *bin_start, *bin_cells, bin_cells_cap;
    int max_bin_count, max_local_nn;
    orc_ranmar rng;
    int step;
    int nev;
    int *ev;                   /* (step, parent, daughter) */
    float syscm[3];            /* the reference's sysCM globals, src/GPUbounce.cu:240 */
    int nfar;
    int *far;                  /* (step, cells not counted) of num_cells_far */
    unsigned err;
    /* pairs used by the last force evaluation (recording mode) */
    int record;
    int *rec[2];
    long nrec[2], reccap[2];
} orc_sys;

/* ------------------------------------------------------------------------ */
/* RANMAR, src/marsaglia.h:54-113 (rmarin) and :115-144 (ranmar).            */
/* ------------------------------------------------------------------------ */
int orc_rmarin(orc_ranmar *r, int ij, int kl)
{
    if (ij < 0 || ij > 31328 || kl < 0 || kl > 30081) return -1;
    int i = (ij / 177) % 177 + 2;
    int j = ij % 177 + 2;
    int k = (kl / 169) % 178 + 1;
    int l = kl % 169;
    for (int ii = 1; ii <= 97; ii++) {
        float s = 0.0f, t = 0.5f;
        for (int jj = 1; jj <= 24; jj++) {
            int m = (((i * j) % 179) * k) % 179;
            i = j; j = k; k = m;
            l = (53 * l + 1) % 169;
            if ((l * m) % 64 >= 32) s += t;
            t *= 0.5f;
        }
        r->u[ii] = s;
    }
    r->c = (float)(362436.0 / 16777216.0);
    r->cd = (float)(7654321.0 / 16777216.0);
    r->cm = (float)(16777213.0 / 16777216.0);
    r->i97 = 97;
    r->j97 = 33;
    r->ok = 1;
    return 0;
}

void orc_ranmar_draw(orc_ranmar *r, float *out, int len)
{
    for (int v = 0; v < len; v++) {
        float uni = r->u[r->i97] - r->u[r->j97];
        if (uni < 0.0f) uni = (float)((double)uni + 1.0);
        r->u[r->i97] = uni;
        if (--r->i97 == 0) r->i97 = 97;
        if (--r->j97 == 0) r->j97 = 97;
        r->c -= r->cd;
        if (r->c < 0.0f) r->c += r->cm;
        uni -= r->c;
        if (uni < 0.0f) uni = (float)((double)uni + 1.0);
        out[v] = uni;
    }
}

/* Seed mapping: src/GPUbounce.cu:1796-1799 (ij = seed, kl = 100*seed) for
 * seeds that the reference accepts; larger seeds are folded into RANMAR's
 * legal range (ij mod 31329, kl mod 30082), the documented extension. */
void orc_seed_map(int seed, int *ij, int *kl)
{
    long s = seed;
    if (s >= 0 && s <= 300) { *ij = (int)s; *kl = (int)(100 * s); return; }
    if (s < 0) s = -s;
    *ij = (int)(s % 31329);
    *kl = (int)((100 * s) % 30082);
}

/* Marsaglia (1972) point on the sphere, src/RandomVector.h:8-24, float. */
void orc_random_vector(orc_ranmar *r, float n[3])
{
    float ran2[2];
    float s;
    do {
        orc_ranmar_draw(r, ran2, 2);
        ran2[0] = 2.0f * ran2[0] - 1.0f;
        ran2[1] = 2.0f * ran2[1] - 1.0f;
        s = ran2[0] * ran2[0] + ran2[1] * ran2[1];
    } while (s >= 1.0f);
    float x1 = ran2[0], x2 = ran2[1];
    n[0] = 2 * x1 * sqrtf(1 - x1 * x1 - x2 * x2);
    n[1] = 2 * x2 * sqrtf(1 - x1 * x1 - x2 * x2);
    n[2] = 1 - 2 * (x1 * x1 + x2 * x2);
}

/* ------------------------------------------------------------------------ */
/* Static data: R0 (src/GPUbounce.cu:1890-1908) and theta0 (:909-938), both  */
/* float on the host from cell 0's initial positions.                        */
/* ------------------------------------------------------------------------ */
static float f3mag(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

void orc_r0_theta0(const float *X, const float *Y, const float *Z, const int *nn,
                   float *r0, float *theta0)
{
    for (int i = 0; i < 180; ++i) {
        for (int k = 0; k < 3; ++k) {
            int N = nn[k * 192 + i];
            r0[k * 192 + i] = f3mag(X[i] - X[N], Y[i] - Y[N], Z[i] - Z[N]);
        }
    }
    for (int n = 0; n < 180; n++) {
        float px = X[n], py = Y[n], pz = Z[n];
        int a = nn[n], b = nn[192 + n], c = nn[384 + n];
        float ix = X[a] - px, iy = Y[a] - py, iz = Z[a] - pz;
        float jx = X[b] - px, jy = Y[b] - py, jz = Z[b] - pz;
        float kx = X[c] - px, ky = Y[c] - py, kz = Z[c] - pz;
        float dij = ix * jx + iy * jy + iz * jz;
        float djk = jx * kx + jy * ky + jz * kz;
        float dik = ix * kx + iy * ky + iz * kz;
        theta0[3 * n + 0] = acosf(dij / (f3mag(ix, iy, iz) * f3mag(jx, jy, jz)));
        theta0[3 * n + 1] = acosf(djk / (f3mag(jx, jy, jz) * f3mag(kx, ky, kz)));
        theta0[3 * n + 2] = acosf(dik / (f3mag(ix, iy, iz) * f3mag(kx, ky, kz)));
    }
}

/* ------------------------------------------------------------------------ */
/* System lifetime                                                           */
/* ------------------------------------------------------------------------ */
orc_sys *orc_create(int cap, const orc_params *P, const orc_topo *T)
{
    orc_sys *s = (orc_sys *)calloc(1, sizeof(orc_sys));
    if (!s) return NULL;
    s->cap = cap;
    s->P = *P;
    s->T = *T;
    size_t nn = (size_t)cap * ORC_SLOTS;
    s->X = calloc(nn, 4); s->Y = calloc(nn, 4); s->Z = calloc(nn, 4);
    s->VX = calloc(nn, 4); s->VY = calloc(nn, 4); s->VZ = calloc(nn, 4);
    s->FC = calloc(3 * nn, 8); s->FD = calloc(3 * nn, 8);
    s->FR = calloc(3 * nn, 4);
    s->CM = calloc(3 * (size_t)cap, 4);
    s->press = calloc(cap, 4); s->E = calloc(cap, 4);
    s->vol = calloc(cap, 4); s->area = calloc(cap, 4);
    s->div_flag = calloc(cap, 1);
    s->aabb = calloc(6 * (size_t)cap, 4);
    s->ev = calloc(3 * ORC_MAX_EVENTS, 4);
    s->far = calloc(2 * ORC_MAX_EVENTS, 4);
    s->syscm[0] = s->syscm[1] = s->syscm[2] = 1.0f;
    return s;
}

void orc_destroy(orc_sys *s)
{
    if (!s) return;
    free(s->X); free(s->Y); free(s->Z); free(s->VX); free(s->VY); free(s->VZ);
    free(s->FC); free(s->FD); free(s->FR); free(s->CM); free(s->press); free(s->E);
    free(s->vol); free(s->area); free(s->div_flag); free(s->aabb);
    free(s->bin_start); free(s->bin_cells); free(s->ev); free(s->far);
    free(s->rec[0]); free(s->rec[1]);
    free(s);
}

/* pointer accessors for the Python wrapper */
float *orc_ptr_f(orc_sys *s, int which)
{
    switch (which) {
    case 0: return s->X; case 1: return s->Y; case 2: return s->Z;
    case 3: return s->VX; case 4: return s->VY; case 5: return s->VZ;
    case 6: return s->CM; case 7: return s->press; case 8: return s->E;
    case 9: return s->vol; case 10: return s->area; case 11: return s->aabb;
    case 12: return s->minmax; case 13: return s->FR; case 14: return s->syscm;
    default: return NULL;
    }
}
double *orc_ptr_d(orc_sys *s, int which) { return which == 0 ? s->FC : s->FD; }
int *orc_ptr_i(orc_sys *s, int which)
{
    switch (which) {
    case 0: return &s->n; case 1: return &s->step; case 2: return &s->xdiv;
    case 3: return &s->nev; case 4: return s->ev;
    case 5: return &s->max_bin_count; case 6: return &s->max_local_nn;
    case 7: return &s->ydiv; case 8: return &s->zdiv;
    case 9: return &s->nfar; case 10: return s->far;
    case 11: return s->bin_start; case 12: return s->bin_cells; case 13: return &s->nbins;
    default: return NULL;
    }
}
unsigned orc_err(orc_sys *s) { return s->err; }
orc_ranmar *orc_rng(orc_sys *s) { return &s->rng; }

/* ------------------------------------------------------------------------ */
/* Centre of mass, src/centermass.cu:8-50.  FP64 sum, stored float.          */
/* ------------------------------------------------------------------------ */
/* FP64 sum of the 180 node values in a fixed association order: six groups
 * of 32 slots (slots 180..191 are zero), each reduced pairwise
 * (w[l] + w[l ^ o] for o = 16, 8, 4, 2, 1), then the six group sums added in
 * order.  This is the order of the CUDA path's warp reduction, so both give
 * the same double before rounding to float. */
static double sum192(const float *v)
{
    double tot = 0.0;
    for (int g = 0; g < 6; ++g) {
        double w[32];
        for (int l = 0; l < 32; ++l) {
            int i = 32 * g + l;
            w[l] = i < 180 ? (double)v[i] : 0.0;
        }
        for (int o = 16; o > 0; o >>= 1) {
            double t[32];
            for (int l = 0; l < 32; ++l) t[l] = w[l] + w[l ^ o];
            for (int l = 0; l < 32; ++l) w[l] = t[l];
        }
        tot += w[0];
    }
    return tot;
}

static void cm_cell(orc_sys *s, int c)
{
    double sx = sum192(s->X + c * 192), sy = sum192(s->Y + c * 192), sz = sum192(s->Z + c * 192);
    s->CM[c] = (float)(sx / 180.0);
    s->CM[s->cap + c] = (float)(sy / 180.0);
    s->CM[2 * s->cap + c] = (float)(sz / 180.0);
}

void orc_center_of_mass(orc_sys *s)
{
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < s->n; ++c) cm_cell(s, c);
}

/* ------------------------------------------------------------------------ */
/* Bounding boxes and global extents, src/propagatebound.cu:10-204,266-323,  */
/* grid divisions src/GPUbounce.cu:1331-1334.  Exact float min/max.          */
/* ------------------------------------------------------------------------ */
static void aabb_cell(orc_sys *s, int c)
{
    const float *X = s->X + c * 192, *Y = s->Y + c * 192, *Z = s->Z + c * 192;
    float a = X[0], b = X[0], cc = Y[0], d = Y[0], e = Z[0], f = Z[0];
    for (int i = 1; i < 180; ++i) {
        if (X[i] < a) a = X[i];
        if (X[i] > b) b = X[i];
        if (Y[i] < cc) cc = Y[i];
        if (Y[i] > d) d = Y[i];
        if (Z[i] < e) e = Z[i];
        if (Z[i] > f) f = Z[i];
    }
    float *bb = s->aabb + 6 * c;
    bb[0] = a; bb[1] = b; bb[2] = cc; bb[3] = d; bb[4] = e; bb[5] = f;
}

static void build_bins(orc_sys *s);

void orc_build_grid(orc_sys *s)
{
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < s->n; ++c) aabb_cell(s, c);
    float mn[3] = {1.0e8f, 1.0e8f, 1.0e8f}, mx[3] = {-1.0e8f, -1.0e8f, -1.0e8f};
    for (int c = 0; c < s->n; ++c) {
        const float *bb = s->aabb + 6 * c;
        for (int d = 0; d < 3; ++d) {
            mn[d] = fminf(mn[d], bb[2 * d]);
            mx[d] = fmaxf(mx[d], bb[2 * d + 1]);
        }
    }
    for (int d = 0; d < 3; ++d) { s->minmax[2 * d] = mn[d]; s->minmax[2 * d + 1] = mx[d]; }
    s->xdiv = (int)((s->minmax[1] - s->minmax[0]) / ORC_DL + 1);
    s->ydiv = (int)((s->minmax[3] - s->minmax[2]) / ORC_DL + 1);
    s->zdiv = (int)((s->minmax[5] - s->minmax[4]) / ORC_DL + 1);
    build_bins(s);
}

static void build_bins(orc_sys *s);

/* Grid divisions and bins from boxes and extents already in place (a state
 * handed over from the CUDA path, whose stale grid is part of the state). */
void orc_rebuild_bins(orc_sys *s)
{
    s->xdiv = (int)((s->minmax[1] - s->minmax[0]) / ORC_DL + 1);
    s->ydiv = (int)((s->minmax[3] - s->minmax[2]) / ORC_DL + 1);
    s->zdiv = (int)((s->minmax[5] - s->minmax[4]) / ORC_DL + 1);
    build_bins(s);
}

/* Cell insertion range of makeNNlist, src/propagatebound.cu:224-241. */
static void bin_range(const orc_sys *s, const float *bb, int lo[3], int hi[3])
{
    float attrac = s->P.att_range;
    int divs[3] = {s->xdiv, s->ydiv, s->zdiv};
    for (int d = 0; d < 3; ++d) {
        float m = s->minmax[2 * d];
        int st = (int)((bb[2 * d] - attrac - m) / ORC_DL);
        if (st < 0) st = 0;
        int en = (int)((bb[2 * d + 1] + attrac - m) / ORC_DL);
        if (en >= divs[d]) en = divs[d] - 1;
        lo[d] = st; hi[d] = en;
    }
}

/* makeNNlist, src/propagatebound.cu:209-263: every cell goes into each bin
 * that its bounding box grown by attraction_range overlaps.  The reference
 * fills bins by atomicAdd (arbitrary order, 32 slots); the oracle fills them
 * in ascending cell order without a cap and flags any bin past 32. */
static void build_bins(orc_sys *s)
{
    long nb = (long)s->xdiv * s->ydiv * s->zdiv;
    if (nb < 1) nb = 1;
    if (nb > 262144) s->err |= ORC_ERR_MEMSET_BUG;
    if (nb > (long)s->nbins) {
        free(s->bin_start);
        s->bin_start = malloc((nb + 1) * sizeof(int));
    }
    s->nbins = (int)nb;
    memset(s->bin_start, 0, (nb + 1) * sizeof(int));
    int lo[3], hi[3];
    for (int c = 0; c < s->n; ++c) {
        bin_range(s, s->aabb + 6 * c, lo, hi);
        for (int x = lo[0]; x <= hi[0]; ++x)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int z = lo[2]; z <= hi[2]; ++z)
                    s->bin_start[z * s->xdiv * s->ydiv + y * s->xdiv + x + 1]++;
    }
    s->max_bin_count = 0;
    for (long b = 0; b < nb; ++b) {
        if (s->bin_start[b + 1] > s->max_bin_count) s->max_bin_count = s->bin_start[b + 1];
        s->bin_start[b + 1] += s->bin_start[b];
    }
    if (s->max_bin_count > 32) s->err |= ORC_ERR_BIN_OVERFLOW;
    int total = s->bin_start[nb];
    if (total > s->bin_cells_cap) {
        free(s->bin_cells);
        s->bin_cells_cap = total + 1024;
        s->bin_cells = malloc(s->bin_cells_cap * sizeof(int));
    }
    int *fill = calloc(nb, sizeof(int));
    for (int c = 0; c < s->n; ++c) {
        bin_range(s, s->aabb + 6 * c, lo, hi);
        for (int x = lo[0]; x <= hi[0]; ++x)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int z = lo[2]; z <= hi[2]; ++z) {
                    int b = z * s->xdiv * s->ydiv + y * s->xdiv + x;
                    s->bin_cells[s->bin_start[b] + fill[b]++] = c;
                }
    }
    free(fill);
}

/* Node bin, src/propagate.cu:360-372 (float, truncation, clamped). */
static int node_bin(const orc_sys *s, float X, float Y, float Z)
{
    int sx = (int)((X - s->minmax[0]) / ORC_DL);
    if (sx < 0) sx = 0;
    if (sx >= s->xdiv) sx = s->xdiv - 1;
    int sy = (int)((Y - s->minmax[2]) / ORC_DL);
    if (sy < 0) sy = 0;
    if (sy >= s->ydiv) sy = s->ydiv - 1;
    int sz = (int)((Z - s->minmax[4]) / ORC_DL);
    if (sz < 0) sz = 0;
    if (sz >= s->zdiv) sz = s->zdiv - 1;
    return sz * s->xdiv * s->ydiv + sy * s->xdiv + sx;
}

/* Bounding-box filter, src/propagate.cu:382-392 (float). Returns 1 if kept. */
/* The squared distance of the reference's contact decisions as its own
 * build evaluates it.  The source writes dx*dx + dy*dy + dz*dz in float
 * (src/propagate.cu:386-390, :418, :614-618, :636); nvcc, with its default
 * floating-point contraction (the reference's makefile does not turn it
 * off), computes it as fmaf(dz, dz, fmaf(dx, dx, dy*dy)).  That association
 * is pinned two ways: a kernel of that expression compiled with the same
 * flags gives this value for every one of 2^20 random inputs, and a pair
 * whose uncontracted value lies at the cut-off and whose contracted value
 * lies above it is left out of the reference's own dissipative force
 * (tests/golden/make_fma_case.py, tests/test_ref_cuda.py). */
static inline float r2_ref(float dx, float dy, float dz)
{
    return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
}

/* Bounding-box filter, src/propagate.cu:382-392.  The box deltas are exact
 * (one of the two terms of each is zero), the sum is r2_ref. */
static int aabb_keep(const float *bb, float X, float Y, float Z, float ra)
{
    float dx = (X - bb[1] > 0.0f) * (X - bb[1]);
    dx += (bb[0] - X > 0.0f) * (bb[0] - X);
    float dy = (Y - bb[3] > 0.0f) * (Y - bb[3]);
    dy += (bb[2] - Y > 0.0f) * (bb[2] - Y);
    float dz = (Z - bb[5] > 0.0f) * (Z - bb[5]);
    dz += (bb[4] - Z > 0.0f) * (bb[4] - Z);
    return !(r2_ref(dx, dy, dz) > ra * ra);
}

/* Accepted neighbour cells of one node (src/propagate.cu:375-404), in bin
 * order. Returns the count. */
static int accepted_cells(const orc_sys *s, int a, float X, float Y, float Z, int *out, int maxout)
{
    int b = node_bin(s, X, Y, Z);
    int cnt = 0;
    for (int k = s->bin_start[b]; k < s->bin_start[b + 1]; ++k) {
        int c = s->bin_cells[k];
        if (c == a) continue;
        if (!aabb_keep(s->aabb + 6 * c, X, Y, Z, s->P.att_range)) continue;
        if (cnt < maxout) out[cnt] = c;
        cnt++;
    }
    return cnt;
}

static inline float pair_r2(float xi, float yi, float zi, float xj, float yj, float zj)
{
    float dx = xi - xj, dy = yi - yj, dz = zi - zj;
    return r2_ref(dx, dy, dz);
}

/* ------------------------------------------------------------------------ */
/* Angle force, src/propagate.cu:26-60, FP64.                                 */
/* ------------------------------------------------------------------------ */
static void angle_force(const double i[3], const double k[3], double theta_o, double kk, double F[3])
{
    double idk = i[0] * k[0] + i[1] * k[1] + i[2] * k[2];
    double ri2 = i[0] * i[0] + i[1] * i[1] + i[2] * i[2];
    double rk2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
    double c1 = -1.0 / sqrt(ri2 * rk2 - idk * idk + 1e-3);
    double c2 = idk / ri2;
    double theta = acos(idk / (sqrt(ri2) * sqrt(rk2) + 1e-3));
    double f = -kk * c1 * (theta - theta_o);
    for (int d = 0; d < 3; ++d) F[d] = f * (k[d] - c2 * i[d]);
}

static void node_pos(const orc_sys *s, int cell, int node, double p[3])
{
    p[0] = s->X[cell * 192 + node];
    p[1] = s->Y[cell * 192 + node];
    p[2] = s->Z[cell * 192 + node];
}

/* NeighNeighs, src/propagate.cu:63-78. */
static void neigh_neighs(const orc_sys *s, int node, int ni, int *nii, int *nij, int *nik,
                         double *t1, double *t2)
{
    const float *th = s->T.theta0 + 3 * ni; /* aij, ajk, aik */
    if (*nii == node) {
        *t1 = th[0]; *t2 = th[2];
        *nii = *nij; *nij = *nik;
    } else if (*nij == node) {
        *t1 = th[0]; *t2 = th[1];
        *nij = *nik;
    } else {
        *t1 = th[2]; *t2 = th[1];
    }
}

/* CalculateAngleForce, src/propagate.cu:81-181, FP64 (k = 1000, :335). */
static void angle_total(const orc_sys *s, int cell, int node, double F[3])
{
    const int *nn = s->T.nn;
    int ni = nn[node], nj = nn[192 + node], nk = nn[384 + node];
    double p[3], pi[3], pj[3], pk[3], a[3], b[3], t[3], u[3];
    node_pos(s, cell, node, p);
    node_pos(s, cell, ni, pi);
    node_pos(s, cell, nj, pj);
    node_pos(s, cell, nk, pk);
    const float *th = s->T.theta0 + 3 * node;
    const double K = 1000.0;
    F[0] = F[1] = F[2] = 0;
    const double *pairs[3][2] = {{pi, pj}, {pj, pk}, {pi, pk}};
    double tho[3] = {th[0], th[1], th[2]};
    for (int q = 0; q < 3; ++q) {
        for (int d = 0; d < 3; ++d) { a[d] = pairs[q][0][d] - p[d]; b[d] = pairs[q][1][d] - p[d]; }
        angle_force(a, b, tho[q], K, t);
        angle_force(b, a, tho[q], K, u);
        for (int d = 0; d < 3; ++d) F[d] -= (t[d] + u[d]);
    }
    int nbr[3] = {ni, nj, nk};
    const double *nbp[3] = {pi, pj, pk};
    for (int q = 0; q < 3; ++q) {
        int n0 = nbr[q];
        int x0 = nn[n0], x1 = nn[192 + n0], x2 = nn[384 + n0];
        double t1, t2;
        neigh_neighs(s, node, n0, &x0, &x1, &x2, &t1, &t2);
        double ti[3], tj[3];
        node_pos(s, cell, x0, ti);
        node_pos(s, cell, x1, tj);
        for (int d = 0; d < 3; ++d) { a[d] = p[d] - nbp[q][d]; b[d] = ti[d] - nbp[q][d]; }
        angle_force(a, b, t1, K, t);
        for (int d = 0; d < 3; ++d) { b[d] = tj[d] - nbp[q][d]; }
        angle_force(a, b, t2, K, u);
        for (int d = 0; d < 3; ++d) F[d] += t[d] + u[d];
    }
}

/* ------------------------------------------------------------------------ */
/* Conservative force, src/propagate.cu:183-520, FP64 values.                */
/* ------------------------------------------------------------------------ */
static void con_force_cell(orc_sys *s, int a, int *max_lnn)
{
    const orc_params *P = &s->P;
    const int cap192 = s->cap * 192;
    double stiff = s->E[a];
    double press = s->press[a];
    double cm[3] = {s->CM[a], s->CM[s->cap + a], s->CM[2 * s->cap + a]};
    const float ra = P->att_range;
    const float ra2 = ra * ra;
    const double rr = P->rep_range;
    const double Ey = P->youngs_mod;
    int lnn[64];
    for (int i = 0; i < 180; ++i) {
        int gi = a * 192 + i;
        float Xf = s->X[gi], Yf = s->Y[gi], Zf = s->Z[gi];
        if (isnan(Xf) || isnan(Yf) || isnan(Zf)) s->err |= ORC_ERR_NAN;
        double x[3] = {Xf, Yf, Zf};
        double F[3] = {0, 0, 0};
        /* springs, :298-314 */
        for (int k = 0; k < 3; ++k) {
            int N = s->T.nn[k * 192 + i];
            double d[3];
            node_pos(s, a, N, d);
            for (int q = 0; q < 3; ++q) d[q] -= x[q];
            double R = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            double R0 = s->T.r0[k * 192 + i];
            for (int q = 0; q < 3; ++q) F[q] += stiff * (R - R0) / R0 * d[q] / R;
        }
        /* internal pressure, :318-330 */
        {
            double r[3] = {x[0] - cm[0], x[1] - cm[1], x[2] - cm[2]};
            double m = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            for (int q = 0; q < 3; ++q) F[q] += 3.0 * press * r[q] / m;
        }
        /* angles, :332-337 */
        if (P->constrain_angles) {
            double t[3];
            angle_total(s, a, i, t);
            for (int q = 0; q < 3; ++q) F[q] += t[q];
        }
        /* contacts, :358-442 */
        int nl = accepted_cells(s, a, Xf, Yf, Zf, lnn, 64);
        if (nl > *max_lnn) *max_lnn = nl;
        if (nl > 64) nl = 64;
        double cf[3] = {0, 0, 0};
        for (int q = 0; q < nl; ++q) {
            int c = lnn[q];
            for (int j = 0; j < 180; ++j) {
                int gj = c * 192 + j;
                float r2 = pair_r2(Xf, Yf, Zf, s->X[gj], s->Y[gj], s->Z[gj]);
                if (r2 >= ra2) continue;
                double d[3] = {x[0] - (double)s->X[gj], x[1] - (double)s->Y[gj], x[2] - (double)s->Z[gj]};
                double R = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                if (R < (double)ra) {
                    double f = -(double)P->att_strength * Ey * ((double)ra - R) / R;
                    for (int w = 0; w < 3; ++w) cf[w] += f * d[w];
                }
                if (R <= rr) {
                    double f = (double)P->rep_strength * Ey * (rr - R) / R;
                    for (int w = 0; w < 3; ++w) cf[w] += f * d[w];
                }
            }
        }
        for (int q = 0; q < 3; ++q) F[q] += cf[q];
        /* rigid box walls, :474-510 (float gap tests) */
        if (P->use_rigid_box) {
            float pos[3] = {Xf, Yf, Zf};
            for (int q = 0; q < 3; ++q) {
                float g1 = pos[q];
                float g2 = P->box[q] - pos[q];
                if (g1 < P->thresh_dist) F[q] += -100.0 * Ey * ((double)g1 - (double)P->thresh_dist);
                if (g2 < P->thresh_dist) F[q] += 100.0 * Ey * ((double)g2 - (double)P->thresh_dist);
            }
        }
        s->FC[gi] = F[0];
        s->FC[cap192 + gi] = F[1];
        s->FC[2 * cap192 + gi] = F[2];
    }
}

void orc_con_force(orc_sys *s)
{
    int mx = 0;
    #pragma omp parallel for schedule(dynamic, 8) reduction(max:mx)
    for (int a = 0; a < s->n; ++a) {
        int m = 0;
        con_force_cell(s, a, &m);
        if (m > mx) mx = m;
    }
    if (mx > s->max_local_nn) s->max_local_nn = mx;
    if (mx > 10) s->err |= ORC_ERR_LOCALNN;
}

/* ------------------------------------------------------------------------ */
/* Dissipative force, src/propagate.cu:523-665, FP64 values.                 */
/* ------------------------------------------------------------------------ */
static void dis_force_cell(orc_sys *s, int a)
{
    const orc_params *P = &s->P;
    const int cap192 = s->cap * 192;
    const float ra = P->att_range;
    const float ra2 = ra * ra;
    int lnn[64];
    for (int i = 0; i < 180; ++i) {
        int gi = a * 192 + i;
        double v[3] = {s->VX[gi], s->VY[gi], s->VZ[gi]};
        double F[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k) {
            int N = s->T.nn[k * 192 + i];
            int gn = a * 192 + N;
            F[0] -= P->gamma_int * (v[0] - (double)s->VX[gn]);
            F[1] -= P->gamma_int * (v[1] - (double)s->VY[gn]);
            F[2] -= P->gamma_int * (v[2] - (double)s->VZ[gn]);
        }
        int N1 = s->T.nn[i], N2 = s->T.nn[192 + i], N3 = s->T.nn[384 + i];
        double p1[3], p2[3], p3[3];
        node_pos(s, a, N1, p1); node_pos(s, a, N2, p2); node_pos(s, a, N3, p3);
        double A[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
        double B[3] = {p3[0] - p1[0], p3[1] - p1[1], p3[2] - p1[2]};
        double nrm[3] = {A[1] * B[2] - A[2] * B[1], A[2] * B[0] - A[0] * B[2], A[0] * B[1] - A[1] * B[0]};
        double m = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        double sg = s->T.sign[i];
        for (int q = 0; q < 3; ++q) nrm[q] = sg * nrm[q] / m;
        float Xf = s->X[gi], Yf = s->Y[gi], Zf = s->Z[gi];
        int nl = accepted_cells(s, a, Xf, Yf, Zf, lnn, 64);
        if (nl > 64) nl = 64;
        for (int q = 0; q < nl; ++q) {
            int c = lnn[q];
            for (int j = 0; j < 180; ++j) {
                int gj = c * 192 + j;
                float r2 = pair_r2(Xf, Yf, Zf, s->X[gj], s->Y[gj], s->Z[gj]);
                if (r2 > ra2) continue;
                double vij[3] = {v[0] - (double)s->VX[gj], v[1] - (double)s->VY[gj], v[2] - (double)s->VZ[gj]};
                double dn = vij[0] * nrm[0] + vij[1] * nrm[1] + vij[2] * nrm[2];
                for (int w = 0; w < 3; ++w) F[w] -= P->gamma_ext * (vij[w] - dn * nrm[w]);
            }
        }
        for (int q = 0; q < 3; ++q) F[q] -= P->gamma_o * v[q];
        s->FD[gi] = F[0];
        s->FD[cap192 + gi] = F[1];
        s->FD[2 * cap192 + gi] = F[2];
    }
}

void orc_dis_force(orc_sys *s)
{
    #pragma omp parallel for schedule(dynamic, 8)
    for (int a = 0; a < s->n; ++a) dis_force_cell(s, a);
}

/* Forces for a subset of cells only (full-size sampled parity). */
void orc_forces_subset(orc_sys *s, const int *cells, int ncells)
{
    int mx = 0;
    #pragma omp parallel for schedule(dynamic, 1) reduction(max:mx)
    for (int q = 0; q < ncells; ++q) {
        int m = 0;
        con_force_cell(s, cells[q], &m);
        dis_force_cell(s, cells[q]);
        if (m > mx) mx = m;
    }
    if (mx > s->max_local_nn) s->max_local_nn = mx;
}

/* ------------------------------------------------------------------------ */
/* Volumes, area, sphericity and the division test, src/volume.cu:5-163.     */
/* ------------------------------------------------------------------------ */
static void volume_cell(orc_sys *s, int c)
{
    double lx[180], ly[180], lz[180];
    double cm[3] = {s->CM[c], s->CM[s->cap + c], s->CM[2 * s->cap + c]};
    for (int i = 0; i < 180; ++i) {
        lx[i] = (double)s->X[c * 192 + i] - cm[0];
        ly[i] = (double)s->Y[c * 192 + i] - cm[1];
        lz[i] = (double)s->Z[c * 192 + i] - cm[2];
    }
    const int *F = s->T.faces;
    double vol = 0, area = 0;
    for (int f = 0; f < 92; ++f) {
        double ax = 0, ay = 0, az = 0;
        for (int i = 0; i < 5; ++i) { ax += lx[F[7 * f + i]]; ay += ly[F[7 * f + i]]; az += lz[F[7 * f + i]]; }
        double fac = (double)0.166666667f;
        if (f < 12) fac = (double)0.2f;
        else { ax += lx[F[7 * f + 5]]; ay += ly[F[7 * f + 5]]; az += lz[F[7 * f + 5]]; }
        ax *= fac; ay *= fac; az *= fac;
        double tv = 0, fa = 0;
        for (int i = 0; i < 6; ++i) {
            int p = F[7 * f + i], q = F[7 * f + i + 1];
            double n1 = (ly[q] * az - ay * lz[q]) * lx[p];
            double n2 = (lz[q] * ax - az * lx[q]) * ly[p];
            double n3 = (lx[q] * ay - ax * ly[q]) * lz[p];
            tv += fabs(n1 + n2 + n3);
            if (s->P.check_sphericity) {
                double x1 = lx[p] - ax, y1 = ly[p] - ay, z1 = lz[p] - az;
                double x2 = lx[q] - ax, y2 = ly[q] - ay, z2 = lz[q] - az;
                double xx = y1 * z2 - z1 * y2, yy = z1 * x2 - x1 * z2, zz = x1 * y2 - y1 * x2;
                fa += 0.5 * sqrt(xx * xx + yy * yy + zz * zz);
            }
        }
        vol += tv;
        area += fa;
    }
    vol = vol / 6.0;
    s->vol[c] = (float)vol;
    if (!isfinite(vol)) { s->err |= ORC_ERR_NONFINITE_VOL; vol = 1.0; }
    int flag = vol > (double)s->P.div_vol;
    if (s->P.check_sphericity) {
        s->area[c] = (float)area;
        double cb = cbrt(vol);
        double psi = 4.835975862049408 * cb * cb / area;
        if (fabs(1.0 - psi) > 0.05) flag = 0;
    }
    s->div_flag[c] = (unsigned char)flag;
}

void orc_volumes(orc_sys *s)
{
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < s->n; ++c) volume_cell(s, c);
}

/* ------------------------------------------------------------------------ */
/* Division, src/postscriptinit.cu:148-256 and src/GPUbounce.cu:1222-1286.   */
/* FP64 half-space geometry, float normal from the bit-exact RNG.            */
/* ------------------------------------------------------------------------ */
static void daughter_positions(orc_sys *s, int parent, int dst, const float nf[3], double sgn,
                               const float *px, const float *py, const float *pz)
{
    double half = (double)(0.5f * s->P.rep_range);
    double n[3] = {sgn * nf[0], sgn * nf[1], sgn * nf[2]};
    double cm[3] = {s->CM[parent], s->CM[s->cap + parent], s->CM[2 * s->cap + parent]};
    double o[3] = {cm[0] + half * n[0], cm[1] + half * n[1], cm[2] + half * n[2]};
    for (int i = 0; i < 180; ++i) {
        double y[3] = {(double)px[i] - o[0], (double)py[i] - o[1], (double)pz[i] - o[2]};
        double dn = y[0] * n[0] + y[1] * n[1] + y[2] * n[2];
        if (dn <= 0.0) { y[0] -= dn * n[0]; y[1] -= dn * n[1]; y[2] -= dn * n[2]; }
        s->X[dst * 192 + i] = (float)(y[0] + o[0]);
        s->Y[dst * 192 + i] = (float)(y[1] + o[1]);
        s->Z[dst * 192 + i] = (float)(y[2] + o[2]);
    }
}

int orc_divide_cell(orc_sys *s, int parent, const float nrm[3])
{
    int nb = s->n;
    if (nb >= s->cap) { s->err |= ORC_ERR_CAPACITY; return -1; }
    float px[180], py[180], pz[180];
    memcpy(px, s->X + parent * 192, 180 * 4);
    memcpy(py, s->Y + parent * 192, 180 * 4);
    memcpy(pz, s->Z + parent * 192, 180 * 4);
    daughter_positions(s, parent, parent, nrm, 1.0, px, py, pz);
    daughter_positions(s, parent, nb, nrm, -1.0, px, py, pz);
    memcpy(s->VX + nb * 192, s->VX + parent * 192, 180 * 4);
    memcpy(s->VY + nb * 192, s->VY + parent * 192, 180 * 4);
    memcpy(s->VZ + nb * 192, s->VZ + parent * 192, 180 * 4);
    s->E[nb] = s->P.daught_same_stiffness ? s->E[parent] : s->P.stiffness1;
    s->press[parent] = s->P.min_p;
    s->press[nb] = s->P.min_p;
    if (s->nev < ORC_MAX_EVENTS) {
        s->ev[3 * s->nev + 0] = s->step;
        s->ev[3 * s->nev + 1] = parent;
        s->ev[3 * s->nev + 2] = nb;
        s->nev++;
    }
    s->n = nb + 1;
    return nb;
}

long orc_pairs(orc_sys *s, int kind, int *out, long maxout);

/* Recording mode: keep the pair sets of the next force evaluations. */
void orc_set_record(orc_sys *s, int on) { s->record = on; }

static void record_pairs(orc_sys *s)
{
    if (!s->record) return;
    for (int k = 0; k < 2; ++k) {
        long cnt = orc_pairs(s, k, NULL, 0);
        if (cnt > s->reccap[k]) {
            free(s->rec[k]);
            s->reccap[k] = cnt + 1024;
            s->rec[k] = malloc(sizeof(int) * 4 * s->reccap[k]);
        }
        s->nrec[k] = orc_pairs(s, k, s->rec[k], s->reccap[k]);
    }
}

long orc_recorded_pairs(orc_sys *s, int kind, int *out, long maxout)
{
    long n = s->nrec[kind];
    if (out) memcpy(out, s->rec[kind], sizeof(int) * 4 * (n < maxout ? n : maxout));
    return n;
}

/* ------------------------------------------------------------------------ */
/* Initialisation up to the first force evaluation, src/GPUbounce.cu:739-763 */
/* and :978-1004 (pressures set to minPressure at :867-871 by the caller).   */
/* ------------------------------------------------------------------------ */
/* CoM correction, src/GPUbounce.cu:1430-1440 (calc_sys_CM :2504-2520 sums
 * the float centres of mass in cell order on the host; CorrectCoMMotion,
 * src/propagate.cu:766-776, shifts the positions only).                     */
static void correct_com(orc_sys *s)
{
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    const int n = s->n, cap = s->cap;
    for (int c = 0; c < n; ++c) {
        sx += s->CM[c];
        sy += s->CM[cap + c];
        sz += s->CM[2 * cap + c];
    }
    sx = sx / (float)n;
    sy = sy / (float)n;
    sz = sz / (float)n;
    s->syscm[0] = sx; s->syscm[1] = sy; s->syscm[2] = sz;
    for (int g = 0; g < n * 192; ++g) {
        s->X[g] -= sx;
        s->Y[g] -= sy;
        s->Z[g] -= sz;
    }
}

/* calc_sys_CM, src/GPUbounce.cu:2504-2520, over the first n cells. */
static void calc_sys_cm(orc_sys *s, int n)
{
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int c = 0; c < n; ++c) {
        sx += s->CM[c];
        sy += s->CM[s->cap + c];
        sz += s->CM[2 * s->cap + c];
    }
    s->syscm[0] = sx / (float)n;
    s->syscm[1] = sy / (float)n;
    s->syscm[2] = sz / (float)n;
}

static float cm_dist2(const orc_sys *s, int c)
{
    float dx = s->CM[c] - s->syscm[0], dy = s->CM[s->cap + c] - s->syscm[1], dz = s->CM[2 * s->cap + c] - s->syscm[2];
    return dx * dx + dy * dy + dz * dz;
}

/* getRmax2, src/GPUbounce.cu:2523-2536. */
static float get_rmax2(const orc_sys *s, int n)
{
    float r2 = 0.0f;
    for (int c = 0; c < n; ++c) {
        float v = cm_dist2(s, c);
        r2 = r2 < v ? v : r2;
    }
    return r2;
}

/* num_cells_far, src/GPUbounce.cu:2538-2565 (called at :1288-1290 after the
 * divisions of a step). */
static int num_cells_far(orc_sys *s, int ndiv)
{
    const int n = s->n;
    if (ndiv == 0 || n < 50) return 0;
    calc_sys_cm(s, n);
    float thr = s->P.far_r * s->P.far_r * get_rmax2(s, n);
    int far = 0;
    for (int c = n - ndiv; c < n; ++c)
        if (cm_dist2(s, c) > thr) ++far;
    return far;
}

/* Cells softened when growth ends, src/GPUbounce.cu:1340-1429. */
static void soften_cells(orc_sys *s)
{
    const orc_params *P = &s->P;
    const int n = s->n;
    int count = P->soft_n;
    if (P->soft_frac > 0) count = (int)roundf(P->soft_frac * (float)n);
    if (P->soft_rand) {
        if (count > n + 1) { s->err |= ORC_ERR_SOFT_CELLS; return; }
        int *chosen = (int *)malloc(sizeof(int) * (count > 0 ? count : 1));
        int got = 0;
        while (got < count) {
            float r;
            orc_ranmar_draw(&s->rng, &r, 1);
            int ind = (int)roundf(r * (float)n);
            int seen = 0;
            for (int q = 0; q < got; ++q)
                if (chosen[q] == ind) { seen = 1; break; }
            if (!seen) chosen[got++] = ind;
        }
        for (int q = 0; q < got; ++q)
            if (chosen[q] < n) s->E[chosen[q]] = P->stiffness2;
        free(chosen);
        return;
    }
    float rmax2 = get_rmax2(s, n);   /* before calc_sys_CM: the previous centre */
    calc_sys_cm(s, n);
    float f = 1.0f - P->closeness;
    for (int c = 0, got = 0; got < count && c < n; ++c)
        if (cm_dist2(s, c) <= f * f * rmax2) { s->E[c] = P->stiffness2; ++got; }
}

/* Initial bond stiffness of the cells, src/GPUbounce.cu:616-692 (centres of
 * mass as everywhere in this oracle, FP64 sums rounded to float). */
int orc_initial_stiffness(const orc_params *P, int rigid, int n, const float *X, const float *Y, const float *Z,
                          orc_ranmar *rng, float *E)
{
    for (int c = 0; c < n; ++c) E[c] = P->stiffness1;
    if (!P->diff_stiff || n == 0) return 0;
    if (P->closeness > 0.f && P->closeness < 1.f) {
        float *m = (float *)malloc(sizeof(float) * 4 * n);
        float sc[3] = {0.f, 0.f, 0.f};
        for (int c = 0; c < n; ++c) {
            m[4 * c] = (float)(sum192(X + c * 192) / 180.0);
            m[4 * c + 1] = (float)(sum192(Y + c * 192) / 180.0);
            m[4 * c + 2] = (float)(sum192(Z + c * 192) / 180.0);
            for (int q = 0; q < 3; ++q) sc[q] += m[4 * c + q];
        }
        float inv = 1.0f / (float)n;   /* float3 / float = (1/a) * b */
        for (int q = 0; q < 3; ++q) sc[q] = inv * sc[q];
        float rmax = 0.f;
        for (int c = 0; c < n; ++c) {
            float dx = m[4 * c] - sc[0], dy = m[4 * c + 1] - sc[1], dz = m[4 * c + 2] - sc[2];
            m[4 * c + 3] = sqrtf(dx * dx + dy * dy + dz * dz);
            if (m[4 * c + 3] > rmax) rmax = m[4 * c + 3];
        }
        for (int c = 0; c < n; ++c)
            if (m[4 * c + 3] / rmax <= P->closeness) E[c] = P->stiffness2;
        free(m);
        return 0;
    }
    int count = P->soft_n;
    if (P->soft_frac > 0.f && P->soft_frac < 1.f) count = (int)roundf(P->soft_frac * (float)n);
    if (count > n) return -1;
    for (int q = 0; q < count; ++q) {
        if (rigid) { E[q] = P->stiffness2; continue; }
        float r;
        orc_ranmar_draw(rng, &r, 1);
        int ind = (int)roundf(r * (float)n);
        if (ind < n) E[ind] = P->stiffness2;
    }
    return 0;
}

void orc_init(orc_sys *s)
{
    s->err = 0;
    orc_center_of_mass(s);
    orc_build_grid(s);
    if (s->P.correct_com) correct_com(s);   /* src/GPUbounce.cu:785-805 */
    record_pairs(s);
    orc_con_force(s);
    orc_dis_force(s);
}

/* ------------------------------------------------------------------------ */
/* Langevin random force, src/propagate.cu:668-678: rand_scale_factor times  */
/* three standard normals per node and step.  The reference draws them from  */
/* curand XORWOW states; the CUDA path (and this restatement of it) from     */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) keyed by rand_seed and  */
/* counted by (node, step), Box-Muller on 24-bit uniforms.                   */
/* ------------------------------------------------------------------------ */
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

static float unit_open(uint32_t r) { return ((float)(r >> 8) + 0.5f) * (1.0f / 16777216.0f); }

void orc_random_force(const orc_params *P, int node, int step, float out[3])
{
    uint32_t c[4] = {(uint32_t)node, (uint32_t)step, 0u, 0u};
    philox4x32_10(c, P->rand_seed, 0x2545F491u);
    float ra = sqrtf(-2.0f * logf(unit_open(c[0]))), ta = 6.28318531f * unit_open(c[1]);
    float rb = sqrtf(-2.0f * logf(unit_open(c[2]))), tb = 6.28318531f * unit_open(c[3]);
    out[0] = P->rand_scale * (ra * cosf(ta));
    out[1] = P->rand_scale * (ra * sinf(ta));
    out[2] = P->rand_scale * (rb * cosf(tb));
}

/* One timestep, src/GPUbounce.cu:1055-1440 (population model disabled).    */
void orc_step(orc_sys *s)
{
    const orc_params *P = &s->P;
    const int cap192 = s->cap * 192;
    const double m = P->mass;
    int step = ++s->step;
    const int N = s->n;
    /* Integrate + ForwardTime, src/propagate.cu:681-763.  The reference keeps
     * forces in float arrays between kernels and evaluates the kick as a float
     * sum scaled in double ("0.5" is a double literal); the drift X + v*dt is
     * one float multiply-add.  Transcribed exactly, so that from the same float
     * state the oracle's positions after the drift are the reference's. */
    const float dtf = P->dt;
    const float rdt = sqrtf(dtf);
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < N; ++c)
        for (int i = 0; i < 180; ++i) {
            int g = c * 192 + i;
            float *V[3] = {s->VX, s->VY, s->VZ};
            float *X[3] = {s->X, s->Y, s->Z};
            for (int q = 0; q < 3; ++q) {
                float fc = (float)s->FC[q * cap192 + g], fd = (float)s->FD[q * cap192 + g];
                float sum = dtf * fc + dtf * fd;
                if (P->add_rands) sum = sum + rdt * s->FR[q * cap192 + g];
                V[q][g] = (float)((double)V[q][g] + 0.5 * (double)sum / m);
                X[q][g] = fmaf(V[q][g], dtf, X[q][g]);
            }
        }
    /* PressureUpdate, src/PressureKernels.cu:4-40 */
    for (int c = 0; c < N; ++c) {
        if (P->diff_stiff && step >= P->phase_count && s->E[c] != P->stiffness1) {
            if (s->press[c] != 0.f) s->press[c] = 0.f;
        } else if (s->press[c] < P->max_p) {
            s->press[c] += P->growth_rate;
        }
    }
    record_pairs(s);
    orc_con_force(s);
    orc_dis_force(s);
    /* CalculateRanForce, src/GPUbounce.cu:1133-1137 */
    if (P->add_rands) {
        #pragma omp parallel for schedule(static)
        for (int c = 0; c < N; ++c)
            for (int i = 0; i < 180; ++i) {
                float fr[3];
                orc_random_force(P, c * 192 + i, step, fr);
                for (int q = 0; q < 3; ++q) s->FR[q * cap192 + c * 192 + i] = fr[q];
            }
    }
    /* VelocityUpdateA/B, src/propagate.cu:714-736 (float forces, double scale) */
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < N; ++c)
        for (int i = 0; i < 180; ++i) {
            int g = c * 192 + i;
            float *V[3] = {s->VX, s->VY, s->VZ};
            for (int q = 0; q < 3; ++q) {
                float fc = (float)s->FC[q * cap192 + g], fd = (float)s->FD[q * cap192 + g];
                float sa = dtf * fc;
                if (P->add_rands) sa = sa + rdt * s->FR[q * cap192 + g];
                V[q][g] = (float)((double)V[q][g] + 0.5 * (double)sa / m);
                V[q][g] = (float)((double)V[q][g] + 0.5 * (double)dtf * (double)fd / m);
            }
        }
    orc_dis_force(s);
    orc_center_of_mass(s);
    if (step <= P->div_time_steps && P->growth_rate > 0) {
        orc_volumes(s);
        int ndiv = 0;
        for (int c = 0; c < N; ++c) {
            if (!s->div_flag[c]) continue;
            s->div_flag[c] = 0;
            float nrm[3];
            orc_random_vector(&s->rng, nrm);
            if (orc_divide_cell(s, c, nrm) < 0) break;
            ++ndiv;
        }
        if (P->far_r > 0) {
            int far = num_cells_far(s, ndiv);
            if (far && s->nfar < ORC_MAX_EVENTS) {
                s->far[2 * s->nfar] = step;
                s->far[2 * s->nfar + 1] = far;
                s->nfar++;
            }
        }
    }
    orc_build_grid(s);
    if (P->diff_stiff && P->soften_after_growth && step == P->div_time_steps + 2) soften_cells(s);
    if (P->correct_com) correct_com(s);
}

void orc_run(orc_sys *s, int nsteps)
{
    for (int k = 0; k < nsteps; ++k) orc_step(s);
}

/* ------------------------------------------------------------------------ */
/* Pair enumeration with the current stale grid: kind 0 = conservative      */
/* (strict cut-off, src/propagate.cu:421), 1 = dissipative (:641).          */
/* Writes (cell_a, node_i, cell_b, node_j) quadruples; returns the count.   */
/* ------------------------------------------------------------------------ */
/* The pairs of cell a's nodes, in node order and then in the accepted-cell
 * order of each node; at most `lim` are written to out (NULL: count only). */
static long pairs_of_cell(const orc_sys *s, int a, int kind, int *out, long lim)
{
    const float ra = s->P.att_range;
    const float ra2 = ra * ra;
    long cnt = 0;
    int lnn[64];
    for (int i = 0; i < 180; ++i) {
        int gi = a * 192 + i;
        float Xf = s->X[gi], Yf = s->Y[gi], Zf = s->Z[gi];
        int nl = accepted_cells(s, a, Xf, Yf, Zf, lnn, 64);
        if (nl > 64) nl = 64;
        for (int q = 0; q < nl; ++q) {
            int c = lnn[q];
            for (int j = 0; j < 180; ++j) {
                int gj = c * 192 + j;
                float r2 = pair_r2(Xf, Yf, Zf, s->X[gj], s->Y[gj], s->Z[gj]);
                int keep = kind == 0 ? (r2 < ra2) : !(r2 > ra2);
                if (!keep) continue;
                if (out && cnt < lim) {
                    out[4 * cnt + 0] = a; out[4 * cnt + 1] = i;
                    out[4 * cnt + 2] = c; out[4 * cnt + 3] = j;
                }
                cnt++;
            }
        }
    }
    return cnt;
}

/* Cells are enumerated in parallel (a count pass, a prefix sum, a fill pass);
 * the output order is the serial order: cell a ascending, then node i, then
 * the accepted cells of the node in bin order, then node j. */
long orc_pairs(orc_sys *s, int kind, int *out, long maxout)
{
    const int n = s->n;
    long *off = (long *)malloc(sizeof(long) * ((size_t)n + 1));
    if (!off) return -1;
    off[0] = 0;
    #pragma omp parallel for schedule(dynamic, 8)
    for (int a = 0; a < n; ++a) off[a + 1] = pairs_of_cell(s, a, kind, NULL, 0);
    for (int a = 0; a < n; ++a) off[a + 1] += off[a];
    const long total = off[n];
    if (out) {
        #pragma omp parallel for schedule(dynamic, 8)
        for (int a = 0; a < n; ++a)
            if (off[a] < maxout) pairs_of_cell(s, a, kind, out + 4 * off[a], maxout - off[a]);
    }
    free(off);
    return total;
}

/* The accepted cells of every node (the cells of the node's stale bin that
 * pass the stale box filter, src/propagate.cu:356-404, uncapped): (cell_a,
 * node_i, cell_c) triples in cell, node, bin order; returns the count. */
static long accepted_of_cell(const orc_sys *s, int a, int *out, long lim)
{
    long cnt = 0;
    int lnn[64];
    for (int i = 0; i < 180; ++i) {
        int gi = a * 192 + i;
        int nl = accepted_cells(s, a, s->X[gi], s->Y[gi], s->Z[gi], lnn, 64);
        if (nl > 64) nl = 64;
        for (int q = 0; q < nl; ++q) {
            if (out && cnt < lim) { out[3 * cnt] = a; out[3 * cnt + 1] = i; out[3 * cnt + 2] = lnn[q]; }
            cnt++;
        }
    }
    return cnt;
}

long orc_accepted(orc_sys *s, int *out, long maxout)
{
    const int n = s->n;
    long *off = (long *)malloc(sizeof(long) * ((size_t)n + 1));
    if (!off) return -1;
    off[0] = 0;
    #pragma omp parallel for schedule(dynamic, 8)
    for (int a = 0; a < n; ++a) off[a + 1] = accepted_of_cell(s, a, NULL, 0);
    for (int a = 0; a < n; ++a) off[a + 1] += off[a];
    const long total = off[n];
    if (out) {
        #pragma omp parallel for schedule(dynamic, 8)
        for (int a = 0; a < n; ++a)
            if (off[a] < maxout) accepted_of_cell(s, a, out + 3 * off[a], maxout - off[a]);
    }
    free(off);
    return total;
}

/* Diagnostic: worst accepted-cell count of any node (the reference keeps at
 * most 10 in localNNs[10], src/propagate.cu:222). */
int orc_max_local_nn(orc_sys *s)
{
    int mx = 0;
    #pragma omp parallel for schedule(static) reduction(max:mx)
    for (int a = 0; a < s->n; ++a)
        for (int i = 0; i < 180; ++i) {
            int lnn[64];
            int gi = a * 192 + i;
            int nl = accepted_cells(s, a, s->X[gi], s->Y[gi], s->Z[gi], lnn, 64);
            if (nl > mx) mx = nl;
        }
    return mx;
}

int orc_sizeof_params(void) { return (int)sizeof(orc_params); }
int orc_sizeof_topo(void) { return (int)sizeof(orc_topo); }
