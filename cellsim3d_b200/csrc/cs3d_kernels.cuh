// cs3d_kernels.cuh -- the per-timestep kernels of libcs3d.so (sm_100a).
//
// One CTA of 192 threads (six warps) owns one cell at a time and walks the
// active cells grid-stride; thread i owns node i.  The cell's 180 positions
// and velocities are staged in shared memory; the 540 bond angles are
// evaluated once each (the reference evaluates every angle twice, from the
// vertex and from the arm end) and their arm-end forces are gathered from
// shared memory in the reference's summation order.
//
// The neighbour list (per cell: candidate cells; per node: the nodes of
// candidate cells within the list radius, as slot << 8 | node) is rebuilt
// on the device whenever the accumulated displacement bound reaches the
// skin, or after a division.  Every step the reference's own contact
// predicates -- stale grid bin of the node, stale bounding box of the
// neighbour cell, strict (conservative) and non-strict (dissipative)
// cut-offs in float -- are evaluated on every list entry, so the contact
// pairs are exactly the reference's.  Partner nodes are read straight from
// global memory: the few hundred partners of a cell stay in L1/L2.
#pragma once
#include "cs3d_dev.cuh"

namespace cs3d {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void atomic_or_err(InstState *st, unsigned bits) { atomicOr(&st->err, bits); }

// Block-wide exclusive scan (NT threads, NT a multiple of 32); wsum[32].
template <int NT>
__device__ __forceinline__ int block_excl_scan(int v, int *wsum, int &total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < NT / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    const int r = (wid > 0 ? wsum[wid - 1] : 0) + x - v;
    total = wsum[NT / 32 - 1];
    __syncthreads();
    return r;
}


// Active cells: the identity for a single instance, else the work table.
__device__ __forceinline__ int n_work(const Dev &d) { return d.single ? d.st[0].n : *d.work_n; }
__device__ __forceinline__ int cell_of(const Dev &d, int w) { return d.single ? w : d.work[w]; }
__device__ __forceinline__ int inst_of(const Dev &d, int a) { return d.single ? 0 : d.cell_inst[a]; }

// Kick of the split velocity Verlet with the reference's mixed precision:
// the float sum is scaled by the double literal 0.5 and divided by the mass
// in double, then stored as float (src/propagate.cu:698-705, 721-723, 732-734).
// a / m, the integrator's division by the particle mass, correctly rounded
// as the IEEE double division the reference evaluates: with im = 1/m
// correctly rounded (set on the host), q = a * im is within one ulp of a/m,
// the remainder a - q m is exact in one FMA, and q + (a - q m) im rounded
// once is the correctly rounded quotient (Markstein's theorem); three FP64
// operations instead of a full division.  Checked against the IEEE division
// on 1.03e9 operand pairs of the integrator's shapes and random masses.
__device__ __forceinline__ double div_m(double a, const InstParams &P)
{
    const double q = a * P.inv_m;
    return fma(fma(-q, P.mass_d, a), P.inv_m, q);
}

// v + 0.5 fsum / m (double arithmetic, stored as float), src/propagate.cu:681-736.
__device__ __forceinline__ float kick(float v, float fsum, const InstParams &P)
{
    return (float)((double)v + div_m(0.5 * (double)fsum, P));
}

// Langevin random force (src/propagate.cu:668-678): rand_scale_factor times
// three standard normals per node and step.  The reference draws them from
// per-node curand XORWOW states; here they come from the counter-based
// Philox4x32-10 generator (Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11; round multipliers and Weyl key
// increments as published there) keyed by the instance's rand_seed and
// counted by (node, step), with the Box-Muller transform on 24-bit uniforms.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ float unit_open(unsigned r)
{
    return ((float)(r >> 8) + 0.5f) * (1.0f / 16777216.0f);  // (0, 1), exact in float
}

__device__ __forceinline__ float3 random_force(const InstParams &P, int a, int i, int step)
{
    const unsigned node = (unsigned)((a - P.base) * SLOTS + i);
    const uint4 r = philox4x32_10(make_uint4(node, (unsigned)step, 0u, 0u), make_uint2(P.rseed, 0x2545F491u));
    const float ra = sqrtf(-2.0f * logf(unit_open(r.x))), ta = 6.28318531f * unit_open(r.y);
    const float rb = sqrtf(-2.0f * logf(unit_open(r.z))), tb = 6.28318531f * unit_open(r.w);
    return make_float3(P.rscale * (ra * cosf(ta)), P.rscale * (ra * sinf(ta)), P.rscale * (rb * cosf(tb)));
}

// 1/sqrt(x), 1/x and sqrt(x) of positive doubles: the hardware's FP64
// approximations (rsqrt.approx.ftz.f64, rcp.approx.ftz.f64; relative error
// below 1e-6 on B200) refined by one Newton step in FP64.  Measured over
// 1e-4..1e4 on B200: relative error below 1.3e-12, far below what the forces
// need (their float rounding is 6e-8), with no float conversions.  The
// arguments are never subnormal (squared lengths of at least ~1e-8).
__device__ __forceinline__ double rsqrt_nr(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y * (1.5 - 0.5 * x * y * y);
}
__device__ __forceinline__ double rcp_nr(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return r * (2.0 - x * r);
}
__device__ __forceinline__ double sqrt_nr(double x)
{
    return x * rsqrt_nr(x);
}

// Bond-angle term for one angle at a vertex with arms P (to the p-end node)
// and Q (to the q-end node); Fp/Fq are GetAngleForce(P, Q) and
// GetAngleForce(Q, P) of src/propagate.cu:26-60 (k = 1000, :335), with the
// same 1e-3 regularisers.  The force is proportional to theta - theta0, a
// difference of two angles near 2 rad whose float rounding alone (1.2e-7)
// would exceed the 1e-5 relative force bar, so it is formed without
// rounding theta.  u = cos(theta) (the reference's regularised ratio) is
// formed in FP64; with c0, s0 = cos, sin of theta0 in FP64,
//   sin(dth / 2) = (c0 - u) / (2 sin(theta0 + dth / 2)),   dth = theta - theta0.
// A float estimate of dth from acosf is refined by one Newton step of this
// equation in FP64 (sin/cos of dth/2 by their Taylor series, |dth/2| < 0.4
// for |dth/2| up to ~1.2 rad), which leaves dth accurate to ~1e-12.
__device__ __forceinline__ void sincos_small(double x, double &s, double &c)
{
    const double x2 = x * x;
    s = x * (1.0 + x2 * (-1.0 / 6 + x2 * (1.0 / 120 + x2 * (-1.0 / 5040 + x2 * (1.0 / 362880 +
            x2 * (-1.0 / 39916800 + x2 * (1.0 / 6227020800.0 - x2 / 1307674368000.0)))))));
    c = 1.0 + x2 * (-0.5 + x2 * (1.0 / 24 + x2 * (-1.0 / 720 + x2 * (1.0 / 40320 + x2 * (-1.0 / 3628800 +
            x2 * (1.0 / 479001600 + x2 * (-1.0 / 87178291200.0 + x2 / 20922789888000.0)))))));
}

// One arm of a vertex: the exact FP64 difference p of two node positions,
// its squared length, length and inverse squared length (from one rsqrt).
struct Arm {
    double x, y, z, r2, len, ir2;
};

__device__ __forceinline__ Arm make_arm(const double3 &to, const double3 &from)
{
    Arm a;
    a.x = to.x - from.x;
    a.y = to.y - from.y;
    a.z = to.z - from.z;
    a.r2 = a.x * a.x + a.y * a.y + a.z * a.z;
    const double r = rsqrt_nr(a.r2);
    a.len = a.r2 * r;
    a.ir2 = r * r;
    return a;
}

// The angle between arms p and q: GetAngleForce(P, Q) (Fp) and
// GetAngleForce(Q, P) (Fq).  |p||q| is the product of the two lengths, as the
// reference forms it (sqrtf(ri_2) * sqrtf(rk_2)).
__device__ __forceinline__ void angle_term(const Arm &p, const Arm &q, float th0f, double c0, double s0, double3 &Fp,
                                           double3 &Fq)
{
    const double idk = p.x * q.x + p.y * q.y + p.z * q.z;
    const double u = idk * rcp_nr(p.len * q.len + 1e-3);
    // float estimate, then one Newton step on g(h) = sin(h) sin(theta0 + h) - (c0 - u)/2, h = dth/2
    double h = 0.5 * (double)(acosf((float)u) - th0f);
    double sh, ch;
    sincos_small(h, sh, ch);
    const double s1 = s0 * ch + c0 * sh, c1t = c0 * ch - s0 * sh;  // sin, cos of theta0 + h
    const double g = sh * s1 - 0.5 * (c0 - u);
    const double dg = ch * s1 + sh * c1t;                            // d/dh of sin(h) sin(theta0 + h)
    h -= g * rcp_nr(dg);
    const double dth = 2.0 * h;
    const double c1 = -rsqrt_nr(p.r2 * q.r2 - idk * idk + 1e-3);
    const double f = -1000.0 * c1 * dth;
    const double cp = idk * p.ir2, cq = idk * q.ir2;
    Fp = make_double3(f * (q.x - cp * p.x), f * (q.y - cp * p.y), f * (q.z - cp * p.z));
    Fq = make_double3(f * (p.x - cq * q.x), f * (p.y - cq * q.y), f * (p.z - cq * q.z));
}

// Shared per-CTA data of the contact sweep: candidate cells with their stale
// boxes and stale insertion bin ranges.
struct SlotData {
    int cell[MAXC];
    float4 lo[MAXC], hi[MAXC];
    short rlo[MAXC][3], rhi[MAXC][3];
    float mn[3];
    int div[3];
};

// Candidate cells and stale grid of cell a (independent loads only, so they
// overlap with the caller's own-node loads; a __syncthreads() follows).
__device__ __forceinline__ void slots_load(const Dev &d, int a, const InstState *st, int par, SlotData &sd)
{
    const int t = threadIdx.x;
    // read in full whatever the count, so that no load waits for another
    // (entries past the count are never used)
    if (t < MAXC) sd.cell[t] = d.cand[(size_t)a * MAXC + t];
    if (t == 0) {
        const int *mm = st->mm[par];
        for (int q = 0; q < 3; ++q) {
            float mn = fminf(o2f(mm[2 * q]), 1.0e8f);
            float mx = fmaxf(o2f(mm[2 * q + 1]), -1.0e8f);
            sd.mn[q] = mn;
            sd.div[q] = grid_div(mn, mx);
        }
    }
}

// Stale boxes / insertion ranges of the candidates (slots_load visible).
__device__ __forceinline__ void slots_boxes(const Dev &d, const InstParams &P, int par, SlotData &sd, int nc)
{
    int t = threadIdx.x;
    if (t < nc) {
        int c = sd.cell[t];
        float4 lo = d.aabb[par][2 * c], hi = d.aabb[par][2 * c + 1];
        sd.lo[t] = lo;
        sd.hi[t] = hi;
        int st, en;
        bin_range_axis(lo.x, hi.x, P.ra, sd.mn[0], sd.div[0], st, en); sd.rlo[t][0] = (short)st; sd.rhi[t][0] = (short)en;
        bin_range_axis(lo.y, hi.y, P.ra, sd.mn[1], sd.div[1], st, en); sd.rlo[t][1] = (short)st; sd.rhi[t][1] = (short)en;
        bin_range_axis(lo.z, hi.z, P.ra, sd.mn[2], sd.div[2], st, en); sd.rlo[t][2] = (short)st; sd.rhi[t][2] = (short)en;
    }
}

// The reference's cell-level contact filter for one node, cached per
// candidate slot (the entries are sorted by slot): the node's stale grid bin
// lies in the slot cell's stale insertion range (the cell is in the node's
// bin list, src/propagatebound.cu:209-256) and the node is within the
// cut-off of the slot cell's stale box (src/propagate.cu:382-392).
struct SlotPred {
    int cur;
    bool ok;
    int nb0, nb1, nb2;
};

__device__ __forceinline__ void pred_init(SlotPred &sp, const SlotData &sd, float3 x)
{
    sp.cur = -1;
    sp.ok = false;
    sp.nb0 = node_bin_axis(x.x, sd.mn[0], sd.div[0]);
    sp.nb1 = node_bin_axis(x.y, sd.mn[1], sd.div[1]);
    sp.nb2 = node_bin_axis(x.z, sd.mn[2], sd.div[2]);
}

__device__ __forceinline__ bool pred_ok(SlotPred &sp, const SlotData &sd, const InstParams &P, float3 x, int s)
{
    if (s != sp.cur) {
        sp.cur = s;
        sp.ok = sp.nb0 >= sd.rlo[s][0] && sp.nb0 <= sd.rhi[s][0] && sp.nb1 >= sd.rlo[s][1] &&
                sp.nb1 <= sd.rhi[s][1] && sp.nb2 >= sd.rlo[s][2] && sp.nb2 <= sd.rhi[s][2] &&
                aabb_keep(sd.lo[s], sd.hi[s], x.x, x.y, x.z, P.ra2);
    }
    return sp.ok;
}

constexpr int EPRE = 8;  // entries prefetched per node at the start of a cell
constexpr int SB = 4;    // entries whose partner loads are in flight together
static_assert(EPRE == 2 * SB && SB == 4, "the sweep's entry window is two batches of four entries");

// ---------------------------------------------------------------------------
// S1 contact sweep of node i over its entries: conservative contact force
// (strict cut-off, src/propagate.cu:406-442) added to F, sum of the velocity
// differences v_i - v_j of the dissipative pairs (non-strict cut-off,
// src/propagate.cu:600-656) in vsum (its tangential part is taken once, by
// tangential()).  Lists the dissipative pairs for S2 (positions do not change
// before S2) and returns their number.
// Partner positions and velocities are read from global memory (L1/L2
// resident: the partners of a cell are a few hundred nodes).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sweep_s1(const Dev &d, const InstParams &P, const SlotData &sd, int a, int i, float3 x,
                                        float3 v, int ne, const uint32_t (&pre)[EPRE / 2], double &FX,
                                        double &FY, double &FZ, double3 &vsum)
{
    const uint16_t *ep = d.ent + (size_t)a * MAXE * SLOTS + i;
    uint16_t *dl = d.dlist + (size_t)a * MAXD * SLOTS + i;
    SlotPred sp;
    pred_init(sp, sd, x);
    int nd = 0;
    // a window of two batches of entries in registers (two per word): the
    // current batch, and the next one, loaded a batch ahead
    uint32_t w0 = pre[0], w1 = pre[1], w2 = pre[2], w3 = pre[3];
    for (int k0 = 0; k0 < ne; k0 += SB) {
        unsigned e[SB];
        e[0] = w0 & 0xffffu;
        e[1] = k0 + 1 < ne ? (w0 >> 16) : 0xffffu;
        e[2] = k0 + 2 < ne ? (w1 & 0xffffu) : 0xffffu;
        e[3] = k0 + 3 < ne ? (w1 >> 16) : 0xffffu;
        w0 = w2;
        w1 = w3;
        {
            const int kn = k0 + 2 * SB;
            unsigned f[SB];
#pragma unroll
            for (int q = 0; q < SB; ++q) f[q] = kn + q < ne ? ep[(size_t)(kn + q) * SLOTS] : 0xffffu;
            w2 = f[0] | (f[1] << 16);
            w3 = f[2] | (f[3] << 16);
        }
        int id[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q) {
            id[q] = -1;
            if (e[q] != 0xffffu && pred_ok(sp, sd, P, x, (int)(e[q] >> 8)))
                id[q] = sd.cell[e[q] >> 8] * SLOTS + (int)(e[q] & 255u);
        }
        float4 xj[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q) xj[q] = id[q] >= 0 ? __ldg(&d.X[id[q]]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int q = 0; q < SB; ++q) {
            if (id[q] < 0) continue;
            const float dx = __fsub_rn(x.x, xj[q].x), dy = __fsub_rn(x.y, xj[q].y), dz = __fsub_rn(x.z, xj[q].z);
            const float r2 = r2_ref(dx, dy, dz);
            if (r2 > P.ra2) { id[q] = -1; continue; }
            if (nd < MAXD) dl[(size_t)nd * SLOTS] = (uint16_t)e[q];
            ++nd;
            if (d.record_pairs) {
                const unsigned long long slot = atomicAdd(d.n_pairs, 1ull);
                if ((long long)slot < d.pair_cap)
                    d.pairs[slot] = make_int4((a << 8) | i, ((id[q] / SLOTS) << 8) | (id[q] % SLOTS),
                                              r2 < P.ra2 ? 3 : 2, 0);
            }
            if (r2 < P.ra2) {
                // distance in FP64 from the exact difference of the float
                // positions: (rr - R) cancels for stiff repulsion
                const double ex = (double)x.x - xj[q].x, ey = (double)x.y - xj[q].y, ez = (double)x.z - xj[q].z;
                const double R2 = ex * ex + ey * ey + ez * ez;
                const double iR = rsqrt_nr(R2);
                const double R = R2 * iR;
                double k = 0.0;
                if (R < (double)P.ra) k += -(double)P.asE * ((double)P.ra - R) * iR;
                if (R <= (double)P.rr) k += (double)P.rsE * ((double)P.rr - R) * iR;
                FX += k * ex;
                FY += k * ey;
                FZ += k * ez;
            }
        }
        float4 vj[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q) vj[q] = id[q] >= 0 ? __ldg(&d.V[id[q]]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int q = 0; q < SB; ++q) {
            if (id[q] < 0) continue;
            // velocity differences of floats are exact in FP64
            vsum.x += (double)v.x - vj[q].x;
            vsum.y += (double)v.y - vj[q].y;
            vsum.z += (double)v.z - vj[q].z;
        }
    }
    return nd;
}

// S2 sweep: sum of the velocity differences over the dissipative pairs found
// by S1 (their list, in column layout), with the velocities after the half
// kicks; tangential() takes its tangential part.
__device__ __forceinline__ double3 sweep_s2(const Dev &d, const int *cell, int a, int i, float3 v, int nd)
{
    const uint16_t *dl = d.dlist + (size_t)a * MAXD * SLOTS + i;
    double3 vt = make_double3(0.0, 0.0, 0.0);
    for (int k0 = 0; k0 < nd; k0 += SB) {
        unsigned e[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q) e[q] = k0 + q < nd ? dl[(size_t)(k0 + q) * SLOTS] : 0xffffu;
        float4 vj[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q)
            vj[q] = e[q] != 0xffffu ? __ldg(&d.Vb[cell[e[q] >> 8] * SLOTS + (int)(e[q] & 255u)])
                                    : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int q = 0; q < SB; ++q) {
            if (e[q] == 0xffffu) continue;
            vt.x += (double)v.x - vj[q].x;
            vt.y += (double)v.y - vj[q].y;
            vt.z += (double)v.z - vj[q].z;
        }
    }
    return vt;
}

// Tangential part of the friction sum, src/propagate.cu:558-656: the
// reference adds v_ij - (v_ij . n) n over the dissipative pairs of node i, with
// n the unit normal of the surface at i, sign * unit((x_N2 - x_N1) x (x_N3 -
// x_N1)).  The projection is linear in v_ij, so the sweeps sum the velocity
// differences alone (S) and this applies it once: S - (S . n) n.  The normal
// is formed in FP64 from exact differences of the float positions.
__device__ __forceinline__ double3 as_d3(const double3 &a) { return a; }
__device__ __forceinline__ double3 as_d3(const float4 &a) { return make_double3(a.x, a.y, a.z); }

// xd: the cell's positions (FP64 copies, or the float4 originals).
template <typename T>
__device__ __forceinline__ double3 tangential(const T *xd, int n0, int n1, int n2, float sgn, double3 S)
{
    const double3 p0 = as_d3(xd[n0]), p1 = as_d3(xd[n1]), p2 = as_d3(xd[n2]);
    const double ax = p1.x - p0.x, ay = p1.y - p0.y, az = p1.z - p0.z;
    const double bx = p2.x - p0.x, by = p2.y - p0.y, bz = p2.z - p0.z;
    const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    const double s = (double)sgn * rsqrt_nr(cx * cx + cy * cy + cz * cz);
    const double nx = s * cx, ny = s * cy, nz = s * cz;
    const double dn = S.x * nx + S.y * ny + S.z * nz;
    return make_double3(S.x - dn * nx, S.y - dn * ny, S.z - dn * nz);
}

// Dissipative force, src/propagate.cu:546-658: bond damping with the three
// neighbours, tangential friction sum vt, viscous drag, on the cell's
// velocities (vd: FP64 copies or the float4 originals).  FP64: the damping
// term is a sum of velocity differences that can cancel.
template <typename T>
__device__ __forceinline__ float3 dis_force(const InstParams &P, const T *vd, int i, int n0, int n1, int n2,
                                           double3 vt)
{
    const double3 v = as_d3(vd[i]);
    double dx = 0.0, dy = 0.0, dz = 0.0;
    const int nbr[3] = {n0, n1, n2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double3 vn = as_d3(vd[nbr[k]]);
        dx += v.x - vn.x; dy += v.y - vn.y; dz += v.z - vn.z;
    }
    const double gi = P.gint, ge = P.gext, go = P.go;
    return make_float3((float)(-gi * dx - ge * vt.x - go * v.x), (float)(-gi * dy - ge * vt.y - go * v.y),
                       (float)(-gi * dz - ge * vt.z - go * v.z));
}

// PressureUpdate, src/PressureKernels.cu:4-40, for the step `step` being
// taken: with variable stiffness, from step phase_count on a cell whose
// stiffness is not stiffness1 has pressure 0; every other cell grows by the
// growth rate up to maxPressure.  The reference runs it after Integrate and
// ForwardTime and before the forces; here S1 applies it to its cell before
// the pressure force (nothing in between reads the pressure), so that the
// stored pressures are always those of the last finished step.
__device__ __forceinline__ float pressure_update(const Dev &d, const InstParams &P, int a, int step)
{
    const float p = d.press[a];
    if (P.diffE && step >= P.phase && d.E[a] != P.stiff1) return 0.0f;
    if (p < P.maxp) return p + P.growth;
    return p;
}

// ---------------------------------------------------------------------------
// K1: first half kick + drift of a step (Integrate + ForwardTime,
// src/propagate.cu:681-763).  The step's PressureUpdate is S1's.
// ---------------------------------------------------------------------------
// One cell, called by the whole block (it synchronises).
__device__ __forceinline__ void integrate_cell(const Dev &d, int a, float *smax)
{
    {
        int inst = inst_of(d, a);
        const InstParams &P = d.prm[inst];
        int i = threadIdx.x;
        float disp = 0.0f;
        if (i < NODES) {
            size_t g = (size_t)a * SLOTS + i;
            float4 x = d.X[g], v = d.V[g], fc = d.FC[g], fd = d.FD[g];
            const float dt = P.dt;
            float sx = __fadd_rn(__fmul_rn(dt, fc.x), __fmul_rn(dt, fd.x));
            float sy = __fadd_rn(__fmul_rn(dt, fc.y), __fmul_rn(dt, fd.y));
            float sz = __fadd_rn(__fmul_rn(dt, fc.z), __fmul_rn(dt, fd.z));
            if (P.rands) {  // + sqrt(dt) Fr of the previous step
                const float4 fr = d.FR[g];
                sx = __fadd_rn(sx, __fmul_rn(P.rdt, fr.x));
                sy = __fadd_rn(sy, __fmul_rn(P.rdt, fr.y));
                sz = __fadd_rn(sz, __fmul_rn(P.rdt, fr.z));
            }
            v.x = kick(v.x, sx, P);
            v.y = kick(v.y, sy, P);
            v.z = kick(v.z, sz, P);
            float4 xn = make_float4(__fmaf_rn(v.x, dt, x.x), __fmaf_rn(v.y, dt, x.y), __fmaf_rn(v.z, dt, x.z), 0.0f);
            // displacement since the last neighbour-list build
            const float4 xb = d.Xb[g];
            float ddx = xn.x - xb.x, ddy = xn.y - xb.y, ddz = xn.z - xb.z;
            disp = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
            d.X[g] = xn;
            d.V[g] = v;
        }
        for (int o = 16; o > 0; o >>= 1) disp = fmaxf(disp, __shfl_xor_sync(0xffffffffu, disp, o));
        if ((i & 31) == 0) smax[i >> 5] = disp;
        __syncthreads();
        if (i == 0) {
            float m = smax[0];
            for (int q = 1; q < SLOTS / 32; ++q) m = fmaxf(m, smax[q]);
            atomicMax(&d.st[inst].disp_step, __float_as_uint(m));
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(SLOTS) k_integrate(Dev d)
{
    const int W = n_work(d);
    __shared__ float smax[SLOTS / 32];
    for (int w = blockIdx.x; w < W; w += gridDim.x) integrate_cell(d, cell_of(d, w), smax);
}

// The next step's half kick and drift of the two cells of each division of
// this step, after their placement (division steps whose S2 did the others).
__global__ void __launch_bounds__(SLOTS) k_integrate_divided(Dev d)
{
    __shared__ float smax[SLOTS / 32];
    const int T = *d.div_total;
    for (int q = blockIdx.x; q < T; q += gridDim.x) {
        const DivEntry e = d.divtab[q];
        integrate_cell(d, e.parent, smax);
        integrate_cell(d, e.daughter, smax);
    }
}

// ---------------------------------------------------------------------------
// Per-step bookkeeping (one block): step counter, rebuild decision, reset of
// the accumulators that this step fills.
// ---------------------------------------------------------------------------
// Hash slices of the list build: every rebuilding instance gets its own
// power-of-two range of buckets (at least its node count), laid out back to
// back; *d.hsz = their total rounded up to whole scan tiles.  Whole block
// (256 threads), after the rebuild decisions.
__device__ void assign_hash_slices(const Dev &d)
{
    __shared__ int wsum[32];
    __shared__ unsigned carry;
    if (threadIdx.x == 0) carry = 0u;
    __syncthreads();
    for (int k0 = 0; k0 < d.n_inst; k0 += 256) {
        const int k = k0 + threadIdx.x;
        int size = 0;
        if (k < d.n_inst) {
            InstState *st = &d.st[k];
            int bits = 0;
            if (st->rebuild) {
                bits = 6;
                while ((1ll << bits) < (long long)st->n * NODES) ++bits;
                size = 1 << bits;
            }
            st->hbits = bits;
        }
        int tot;
        const int off = block_excl_scan<256>(size, wsum, tot);
        if (k < d.n_inst) d.st[k].hbase = carry + (unsigned)off;
        if (threadIdx.x == 0) carry += (unsigned)tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        unsigned h = (carry + SCAN_TILE - 1) / SCAN_TILE * SCAN_TILE;
        *d.hsz = (int)(h < (unsigned)SCAN_TILE ? (unsigned)SCAN_TILE : h);
    }
}

__global__ void __launch_bounds__(256) k_step_begin(Dev d, int par_next)
{
    __shared__ int any;
    if (threadIdx.x == 0) { any = 0; *d.div_total = 0; }
    __syncthreads();
    for (int k = threadIdx.x; k < d.n_inst; k += blockDim.x) {
        InstState *st = &d.st[k];
        const InstParams &P = d.prm[k];
        st->step += 1;
        // ds: the largest distance of any node from its anchor (Xb, its
        // position at a build).  Every list built at time tb with radius
        // ra + skin + 2*ds(tb) stays complete while all nodes stay within
        // skin/2 of their anchors: a pair within ra now was within
        // ra + 2*(skin/2 + ds(tb)) at tb.  Whole-instance builds (ds reset
        // to 0) use ra + skin; the 1e-3 slack covers float rounding.
        // After divisions, only the divided cells (anchors reset) and the
        // cells within the list radius of them are rebuilt, unless ds is
        // already large.
        const float ds = __uint_as_float(st->disp_step);
        st->disp_step = 0u;
        if (P.sk_n > 0) {
            // the skin of the instance's population range; a change is a
            // whole-instance rebuild with the new list radius
            float want = P.skin_base;
            for (int q = 0; q < P.sk_n; ++q)
                if (st->n >= P.sk_min[q]) want = P.sk_val[q];
            if (want != P.skin) {
                InstParams *Pw = &d.prm[k];
                Pw->skin = want;
                Pw->rlist = Pw->ra + want;
                st->force_rebuild = 1;
            }
        }
        const bool by_disp = st->force_rebuild || !(2.0f * ds + 1e-3f < P.skin);
        const bool by_div = st->div_count > 0 && ds > 0.25f * P.skin;
        const bool full = by_disp || by_div;
        if (by_div && !by_disp) st->rebuilds_div += 1;
        const bool part = !full && st->div_count > 0;
        st->rebuild = full ? 2 : part ? 1 : 0;
        st->rcur = full ? P.rlist : P.rlist + 2.0f * ds + 1e-3f;
        st->force_rebuild = 0;
        st->div_count = 0;
        if (full || part) {
            if (full) st->rebuilds += 1;
            any = 1;
        }
        for (int q = 0; q < 3; ++q) {
            st->mm[par_next][2 * q] = f2o(1.0e30f);
            st->mm[par_next][2 * q + 1] = f2o(-1.0e30f);
        }
    }
    __syncthreads();
    assign_hash_slices(d);
    if (threadIdx.x == 0) {
        d.flags[0] = any;
        *d.n_pairs = 0ull;
    }
}

// Whole-instance list rebuild of every instance at the next step.
__global__ void k_force_rebuild(Dev d)
{
    for (int k = threadIdx.x; k < d.n_inst; k += blockDim.x) d.st[k].force_rebuild = 1;
}

// Init variant: rebuild everything, reset the grid accumulators.
__global__ void __launch_bounds__(256) k_init_begin(Dev d)
{
    for (int k = threadIdx.x; k < d.n_inst; k += blockDim.x) {
        InstState *st = &d.st[k];
        st->rebuild = 2;
        st->rcur = d.prm[k].rlist;
        st->force_rebuild = 0;
        st->disp_step = 0u;
        for (int p = 0; p < 2; ++p)
            for (int q = 0; q < 3; ++q) {
                st->mm[p][2 * q] = f2o(1.0e30f);
                st->mm[p][2 * q + 1] = f2o(-1.0e30f);
            }
    }
    __syncthreads();
    assign_hash_slices(d);
    if (threadIdx.x == 0) {
        d.flags[0] = 1;
        *d.div_total = 0;
        *d.n_pairs = 0ull;
    }
}

// ---------------------------------------------------------------------------
// Block reductions over the 180 nodes of a cell.
// ---------------------------------------------------------------------------
struct GeomScratch {
    double sum[SLOTS / 32][3];
    float mn[SLOTS / 32][3], mx[SLOTS / 32][3];
    double vol[SLOTS / 32], area[SLOTS / 32];
    double fc[CS3D_FACES][3];   // face centres relative to the cell's centre of mass
};

// Centre of mass (FP64 sum, src/centermass.cu:8-50) and bounding box
// (src/propagatebound.cu:10-141) of the cell staged in xs.
__device__ __forceinline__ void cell_geom(const float4 *xs, GeomScratch &gs, float3 &cm, float4 &lo, float4 &hi)
{
    int i = threadIdx.x, w = i >> 5, l = i & 31;
    double sx = 0, sy = 0, sz = 0;
    float mnx = 1e30f, mny = 1e30f, mnz = 1e30f, mxx = -1e30f, mxy = -1e30f, mxz = -1e30f;
    if (i < NODES) {
        float4 p = xs[i];
        sx = p.x; sy = p.y; sz = p.z;
        mnx = mxx = p.x; mny = mxy = p.y; mnz = mxz = p.z;
    }
    sx = warp_sum(sx); sy = warp_sum(sy); sz = warp_sum(sz);
    for (int o = 16; o > 0; o >>= 1) {
        mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mnz = fminf(mnz, __shfl_xor_sync(0xffffffffu, mnz, o));
        mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        mxz = fmaxf(mxz, __shfl_xor_sync(0xffffffffu, mxz, o));
    }
    if (l == 0) {
        gs.sum[w][0] = sx; gs.sum[w][1] = sy; gs.sum[w][2] = sz;
        gs.mn[w][0] = mnx; gs.mn[w][1] = mny; gs.mn[w][2] = mnz;
        gs.mx[w][0] = mxx; gs.mx[w][1] = mxy; gs.mx[w][2] = mxz;
    }
    __syncthreads();
    double tx = 0, ty = 0, tz = 0;
    float a0 = 1e30f, a1 = 1e30f, a2 = 1e30f, b0 = -1e30f, b1 = -1e30f, b2 = -1e30f;
    for (int q = 0; q < SLOTS / 32; ++q) {
        tx += gs.sum[q][0]; ty += gs.sum[q][1]; tz += gs.sum[q][2];
        a0 = fminf(a0, gs.mn[q][0]); a1 = fminf(a1, gs.mn[q][1]); a2 = fminf(a2, gs.mn[q][2]);
        b0 = fmaxf(b0, gs.mx[q][0]); b1 = fmaxf(b1, gs.mx[q][1]); b2 = fmaxf(b2, gs.mx[q][2]);
    }
    cm = make_float3((float)(tx / 180.0), (float)(ty / 180.0), (float)(tz / 180.0));
    lo = make_float4(a0, a1, a2, 0.0f);
    hi = make_float4(b0, b1, b2, 0.0f);
}

// Volume, area and the division test, src/volume.cu:5-163, in FP64.  Each
// face (12 pentagons, 80 hexagons, vertices relative to the cell's centre of
// mass) is cut into triangles at its vertex average; the volume is the sum
// of |det| / 6 of the tetrahedra (centre of mass, triangle) and the area the
// sum of the triangle areas.  The face centres first (one thread per face),
// then the 552 triangles dealt out to all threads.
__device__ __noinline__ void cell_volume(const Dev &d, const float4 *xs, float3 cm, GeomScratch &gs, bool sph,
                                         double &vol, double &area)
{
    const int t = threadIdx.x, w = t >> 5, l = t & 31;
    const double cx = cm.x, cy = cm.y, cz = cm.z;
    if (t < CS3D_FACES) {
        const uint8_t *F = d.topo.faces + 7 * t;
        double ax = 0, ay = 0, az = 0;
        for (int q = 0; q < 5; ++q) {
            const float4 p = xs[F[q]];
            ax += (double)p.x - cx; ay += (double)p.y - cy; az += (double)p.z - cz;
        }
        double fac = (double)0.166666667f;
        if (t < 12) fac = (double)0.2f;
        else {
            const float4 p = xs[F[5]];
            ax += (double)p.x - cx; ay += (double)p.y - cy; az += (double)p.z - cz;
        }
        gs.fc[t][0] = ax * fac; gs.fc[t][1] = ay * fac; gs.fc[t][2] = az * fac;
    }
    __syncthreads();
    double tv = 0, fa = 0;
    for (int k = t; k < CS3D_FACES * 6; k += SLOTS) {
        const int f = k / 6, q = k - 6 * f;
        const uint8_t *F = d.topo.faces + 7 * f;
        const float4 p0 = xs[F[q]], p1 = xs[F[q + 1]];
        const double x0 = (double)p0.x - cx, y0 = (double)p0.y - cy, z0 = (double)p0.z - cz;
        const double x1 = (double)p1.x - cx, y1 = (double)p1.y - cy, z1 = (double)p1.z - cz;
        const double ax = gs.fc[f][0], ay = gs.fc[f][1], az = gs.fc[f][2];
        const double n1 = (y1 * az - ay * z1) * x0;
        const double n2 = (z1 * ax - az * x1) * y0;
        const double n3 = (x1 * ay - ax * y1) * z0;
        tv += fabs(n1 + n2 + n3);
        if (sph) {
            const double u1 = x0 - ax, v1 = y0 - ay, w1 = z0 - az;
            const double u2 = x1 - ax, v2 = y1 - ay, w2 = z1 - az;
            const double xx = v1 * w2 - w1 * v2, yy = w1 * u2 - u1 * w2, zz = u1 * v2 - v1 * u2;
            fa += 0.5 * sqrt(xx * xx + yy * yy + zz * zz);
        }
    }
    tv = warp_sum(tv);
    fa = warp_sum(fa);
    if (l == 0) { gs.vol[w] = tv; gs.area[w] = fa; }
    __syncthreads();
    vol = 0; area = 0;
    for (int q = 0; q < SLOTS / 32; ++q) { vol += gs.vol[q]; area += gs.area[q]; }
    vol = vol / 6.0;
}

// ---------------------------------------------------------------------------
// S1: conservative force (src/propagate.cu:183-520), first dissipative force
// (:523-665 with v after Integrate) and VelocityUpdateA/B (:714-736).
// INIT = true evaluates the initial forces of src/GPUbounce.cu:978-1004
// (no velocity update; Fd written to FD).
// ---------------------------------------------------------------------------
// Arm forces of the angles at each vertex, summed by destination: entry
// vertex*3 + k goes to the vertex's k-th neighbour.
struct ArmForces {
    double x[SLOTS * 3], y[SLOTS * 3], z[SLOTS * 3];
};

struct S1Smem {
    double3 xd[SLOTS];   // FP64 copies of the positions and velocities: the
    double3 vd[SLOTS];   // FP64 terms read them without conversions
    SlotData sd;
    ArmForces arm;
    float press;         // the cell's pressure of this step
};

template <bool INIT>
__global__ void __launch_bounds__(SLOTS, 4) k_s1(Dev d, int par)
{
    extern __shared__ __align__(16) unsigned char s1_raw[];  // sizeof(S1Smem), > 48 KB
    S1Smem &sm = *reinterpret_cast<S1Smem *>(s1_raw);
    const int W = n_work(d);
    const int i = threadIdx.x;
    const uint32_t nnp = (i < NODES) ? __ldg(&d.topo.nnpack[i]) : 0u;
    const int n0 = nnp & 255, n1 = (nnp >> 8) & 255, n2 = (nnp >> 16) & 255;
    const float sgn = (float)(int8_t)(nnp >> 24);
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = cell_of(d, w);
        const int inst = inst_of(d, a);
        const InstParams &P = d.prm[inst];
        const size_t g = (size_t)a * SLOTS + i;
        const int nc = d.ncand[a];
        float4 x4 = make_float4(0, 0, 0, 0), v4 = make_float4(0, 0, 0, 0);
        if (i < NODES) { x4 = d.X[g]; v4 = d.V[g]; }
        const int ne = d.nent[g];
        uint32_t pre[EPRE / 2];
#pragma unroll
        for (int q = 0; q < EPRE / 2; ++q)
            pre[q] = (uint32_t)d.ent[((size_t)a * MAXE + 2 * q) * SLOTS + i] |
                     ((uint32_t)d.ent[((size_t)a * MAXE + 2 * q + 1) * SLOTS + i] << 16);
        sm.xd[i] = make_double3(x4.x, x4.y, x4.z);
        sm.vd[i] = make_double3(v4.x, v4.y, v4.z);
        slots_load(d, a, &d.st[inst], par, sm.sd);
        if (i == 0) {
            // this step's PressureUpdate (none before the initial forces)
            const float pr = INIT ? d.press[a] : pressure_update(d, P, a, d.st[inst].step);
            if (!INIT) d.press[a] = pr;
            sm.press = pr;
        }
        __syncthreads();
        slots_boxes(d, P, par, sm.sd, nc);
        const float3 x = f3(x4);
        const float3 v = f3(v4);
        // bond angles: thread = vertex, three angles each
        if (P.angles && i < NODES) {
            const double3 xi = sm.xd[i];
            const Arm pa = make_arm(sm.xd[n0], xi), pb = make_arm(sm.xd[n1], xi), pc = make_arm(sm.xd[n2], xi);
            const double2 *cs0 = d.topo.cs0 + 3 * i;
            const float4 th = __ldg(&d.topo.th0[i]);
            // angles (n0, n1), (n1, n2), (n0, n2); arm ends summed by destination
            double3 F01p, F01q, F12p, F12q, F02p, F02q;
            double2 t0 = __ldg(&cs0[0]);
            angle_term(pa, pb, th.x, t0.x, t0.y, F01p, F01q);
            t0 = __ldg(&cs0[1]);
            angle_term(pb, pc, th.y, t0.x, t0.y, F12p, F12q);
            t0 = __ldg(&cs0[2]);
            angle_term(pa, pc, th.z, t0.x, t0.y, F02p, F02q);
            const int o = i * 3;
            sm.arm.x[o] = F01p.x + F02p.x; sm.arm.y[o] = F01p.y + F02p.y; sm.arm.z[o] = F01p.z + F02p.z;
            sm.arm.x[o + 1] = F01q.x + F12p.x; sm.arm.y[o + 1] = F01q.y + F12p.y; sm.arm.z[o + 1] = F01q.z + F12p.z;
            sm.arm.x[o + 2] = F12q.x + F02q.x; sm.arm.y[o + 2] = F12q.y + F02q.y; sm.arm.z[o + 2] = F12q.z + F02q.z;
        }
        __syncthreads();
        if (i < NODES) {
            // The node force is accumulated in FP64: its terms (pressure up
            // to ~1e3, stiff contact repulsion up to ~1e4) can cancel to a
            // net force orders of magnitude smaller, and the sum is rounded to
            // float once, as the reference stores it.
            double FX = 0.0, FY = 0.0, FZ = 0.0;
            if (isnan(x.x) || isnan(x.y) || isnan(x.z)) atomic_or_err(&d.st[inst], CS3D_ERRBIT_NAN);
            // springs, src/propagate.cu:298-314:
            // k (R - R0) / R0 * d / R = k (1/R0 - 1/R) d
            const double stiff = d.E[a];
            const int nbr[3] = {n0, n1, n2};
            const double3 xi = sm.xd[i];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                // exact FP64 differences of the float positions
                const double3 xn = sm.xd[nbr[k]];
                const double ex = xn.x - xi.x, ey = xn.y - xi.y, ez = xn.z - xi.z;
                const double iR = rsqrt_nr(ex * ex + ey * ey + ez * ez);
                const double c = stiff * (__ldg(&d.topo.r0i[3 * i + k]) - iR);
                FX += c * ex; FY += c * ey; FZ += c * ez;
            }
            // internal pressure, src/propagate.cu:318-330 (CM of the previous step)
            {
                const float4 cm = d.CM[a];
                const double rx = xi.x - cm.x, ry = xi.y - cm.y, rz = xi.z - cm.z;
                const double c = 3.0 * (double)sm.press * rsqrt_nr(rx * rx + ry * ry + rz * rz);
                FX += c * rx; FY += c * ry; FZ += c * rz;
            }
            // bond angles, src/propagate.cu:81-181: the vertex terms (minus
            // the arm forces of the angles at i) and the arm terms (the arm
            // forces that the angles at the three neighbours send to i)
            if (P.angles) {
                const int o = i * 3;
                const uint4 am = __ldg(&d.topo.arm[i]);
                FX += sm.arm.x[am.x] + sm.arm.x[am.y] + sm.arm.x[am.z] - (sm.arm.x[o] + sm.arm.x[o + 1] + sm.arm.x[o + 2]);
                FY += sm.arm.y[am.x] + sm.arm.y[am.y] + sm.arm.y[am.z] - (sm.arm.y[o] + sm.arm.y[o + 1] + sm.arm.y[o + 2]);
                FZ += sm.arm.z[am.x] + sm.arm.z[am.y] + sm.arm.z[am.z] - (sm.arm.z[o] + sm.arm.z[o + 1] + sm.arm.z[o + 2]);
            }
            // contacts, src/propagate.cu:356-442 and the first dissipative sweep
            double3 vsum = make_double3(0.0, 0.0, 0.0);
            const int nd = sweep_s1(d, P, sm.sd, a, i, x, v, ne, pre, FX, FY, FZ, vsum);
            const double3 vt = tangential(sm.xd, n0, n1, n2, sgn, vsum);
            if (nd > MAXD) atomic_or_err(&d.st[inst], CS3D_ERRBIT_ENTRY_OVERFLOW);
            // rigid box walls, src/propagate.cu:474-510 (float gap tests)
            if (P.rigid) {
                const double wk = P.wallk, th = P.thresh;
                float g1 = x.x, g2 = __fsub_rn(P.box[0], x.x);
                if (g1 < P.thresh) FX += -wk * ((double)g1 - th);
                if (g2 < P.thresh) FX += wk * ((double)g2 - th);
                g1 = x.y; g2 = __fsub_rn(P.box[1], x.y);
                if (g1 < P.thresh) FY += -wk * ((double)g1 - th);
                if (g2 < P.thresh) FY += wk * ((double)g2 - th);
                g1 = x.z; g2 = __fsub_rn(P.box[2], x.z);
                if (g1 < P.thresh) FZ += -wk * ((double)g1 - th);
                if (g2 < P.thresh) FZ += wk * ((double)g2 - th);
            }
            const float3 fd = dis_force(P, sm.vd, i, n0, n1, n2, vt);
            d.FC[g] = make_float4((float)FX, (float)FY, (float)FZ, 0.f);
            d.ndis[g] = (uint8_t)(nd < MAXD ? nd : MAXD);
            if (INIT) {
                d.FD[g] = make_float4(fd.x, fd.y, fd.z, 0.f);
                d.FR[g] = make_float4(0.f, 0.f, 0.f, 0.f);  // no random force before the first step
            } else {
                const float dt = P.dt;
                // random force of this step (CalculateRanForce, GPUbounce.cu:1133-1137)
                float3 fr = make_float3(0.f, 0.f, 0.f);
                if (P.rands) {
                    fr = random_force(P, a, i, d.st[inst].step);
                    d.FR[g] = make_float4(fr.x, fr.y, fr.z, 0.f);
                }
                // VelocityUpdateA reads the stored (float) conservative force:
                // 0.5 (dt Fc + sqrt(dt) Fr) / m
                float vx = kick(v.x, __fadd_rn(__fmul_rn(dt, (float)FX), __fmul_rn(P.rdt, fr.x)), P);
                float vy = kick(v.y, __fadd_rn(__fmul_rn(dt, (float)FY), __fmul_rn(P.rdt, fr.y)), P);
                float vz = kick(v.z, __fadd_rn(__fmul_rn(dt, (float)FZ), __fmul_rn(P.rdt, fr.z)), P);
                const double hdt = 0.5 * (double)dt;
                vx = (float)((double)vx + div_m(hdt * (double)fd.x, P));
                vy = (float)((double)vy + div_m(hdt * (double)fd.y, P));
                vz = (float)((double)vz + div_m(hdt * (double)fd.z, P));
                d.Vb[g] = make_float4(vx, vy, vz, 0.f);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// S2: second dissipative force with the updated velocities
// (src/GPUbounce.cu:1151), centre of mass (:1164), volumes and division
// flags (:1172, DIV only), bounding boxes and grid extents for the next step
// (:1312-1334).  The dissipative pairs are those S1 listed (same positions).
// ---------------------------------------------------------------------------
struct S2Smem {
    float4 xs[SLOTS];
    float4 vs[SLOTS];
    int cell[MAXC];

    GeomScratch gs;
    int dflag;   // the cell divides (division steps)
};

// Integrate + ForwardTime of the next step (src/propagate.cu:681-763) on the
// node's force and velocity after this step; returns the node's distance from
// its list anchor.  The same operations as k_integrate.
__device__ __forceinline__ float next_kick(const Dev &d, const InstParams &P, size_t g, float4 x4, float4 v4,
                                           float3 fd)
{
    const float4 fc = d.FC[g];
    const float dt = P.dt;
    float sx = __fadd_rn(__fmul_rn(dt, fc.x), __fmul_rn(dt, fd.x));
    float sy = __fadd_rn(__fmul_rn(dt, fc.y), __fmul_rn(dt, fd.y));
    float sz = __fadd_rn(__fmul_rn(dt, fc.z), __fmul_rn(dt, fd.z));
    if (P.rands) {
        const float4 fr = d.FR[g];
        sx = __fadd_rn(sx, __fmul_rn(P.rdt, fr.x));
        sy = __fadd_rn(sy, __fmul_rn(P.rdt, fr.y));
        sz = __fadd_rn(sz, __fmul_rn(P.rdt, fr.z));
    }
    float4 vn = v4;
    vn.x = kick(v4.x, sx, P);
    vn.y = kick(v4.y, sy, P);
    vn.z = kick(v4.z, sz, P);
    const float4 xn = make_float4(__fmaf_rn(vn.x, dt, x4.x), __fmaf_rn(vn.y, dt, x4.y),
                                  __fmaf_rn(vn.z, dt, x4.z), 0.0f);
    const float4 xb = d.Xb[g];
    const float ddx = xn.x - xb.x, ddy = xn.y - xb.y, ddz = xn.z - xb.z;
    d.X[g] = xn;
    d.V[g] = vn;
    return sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
}

__device__ __forceinline__ void flush_mm(Dev &d, int inst, int pn, const float *acc)
{
    int *mm = d.st[inst].mm[pn];
    for (int q = 0; q < 3; ++q) {
        atomicMin(&mm[2 * q], f2o(acc[2 * q]));
        atomicMax(&mm[2 * q + 1], f2o(acc[2 * q + 1]));
    }
}

// FUSE: the first half kick and drift of the next step (k_integrate) are
// done here, on the force and velocity in registers: FUSE 1 when the next
// step follows in the same launch sequence, FUSE 2 on the last step of a
// cs3d_step call, which also keeps the step-end positions (Xe; the step-end
// velocities are Vb) for the state read-back, so that the next call starts
// without a k_integrate pass.
template <bool DIV, int FUSE>
__global__ void __launch_bounds__(SLOTS, 5) k_s2(Dev d, int par)
{
    __shared__ S2Smem sm;
    __shared__ float smax[SLOTS / 32];
    const int W = n_work(d);
    const int i = threadIdx.x;
    const int pn = par ^ 1;
    const uint32_t nnp = (i < NODES) ? __ldg(&d.topo.nnpack[i]) : 0u;
    const int n0 = nnp & 255, n1 = (nnp >> 8) & 255, n2 = (nnp >> 16) & 255;
    const float sgn = (float)(int8_t)(nnp >> 24);
    int acc_inst = -1;
    float acc[6];
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = cell_of(d, w);
        const int inst = inst_of(d, a);
        const InstParams &P = d.prm[inst];
        InstState *st = &d.st[inst];
        const size_t g = (size_t)a * SLOTS + i;
        float4 x4 = make_float4(0, 0, 0, 0), v4 = make_float4(0, 0, 0, 0);
        int nd = 0;
        if (i < NODES) { x4 = d.X[g]; v4 = d.Vb[g]; nd = d.ndis[g]; }
        if (i < MAXC) sm.cell[i] = d.cand[(size_t)a * MAXC + i];
        sm.xs[i] = x4;
        sm.vs[i] = v4;
        __syncthreads();
        float disp = 0.0f;

        float3 fdk = make_float3(0.f, 0.f, 0.f);
        if (i < NODES) {
            const float3 v = f3(v4);
            const double3 vt = tangential(sm.xs, n0, n1, n2, sgn, sweep_s2(d, sm.cell, a, i, v, nd));
            const float3 fd = dis_force(P, sm.vs, i, n0, n1, n2, vt);

            d.FD[g] = make_float4(fd.x, fd.y, fd.z, 0.f);
            fdk = fd;
            if (FUSE == 2 && !DIV) d.Xe[g] = x4;
            if (FUSE && !DIV) disp = next_kick(d, P, g, x4, v4, fd);
            else d.V[g] = v4;
        }
        if (FUSE && !DIV) {
            for (int o = 16; o > 0; o >>= 1) disp = fmaxf(disp, __shfl_xor_sync(0xffffffffu, disp, o));
            if ((i & 31) == 0) smax[i >> 5] = disp;
        }
        if (i == 0) sm.dflag = 0;
        float3 cm;
        float4 lo, hi;
        cell_geom(sm.xs, sm.gs, cm, lo, hi);
        if (DIV) {
            if (st->step <= P.div_steps && P.growth > 0.0f) {
                double vol, area;
                cell_volume(d, sm.xs, cm, sm.gs, P.check_sph != 0, vol, area);
                if (i == 0) {
                    d.vol[a] = (float)vol;
                    if (!isfinite(vol)) { atomic_or_err(st, CS3D_ERRBIT_NONFINITE_VOL); vol = 1.0; }
                    int flag = vol > (double)P.divvol;
                    if (P.check_sph) {
                        d.area[a] = (float)area;
                        double cb = cbrt(vol);
                        double psi = 4.835975862049408 * cb * cb / area;
                        if (fabs(1.0 - psi) > 0.05) flag = 0;
                    }
                    d.divflag[a] = (uint8_t)flag;
                    sm.dflag = flag;
                }
            }
        }
        if (FUSE && DIV) {
            // With the division decision known: a cell that does not divide
            // takes the next step's half kick and drift here, the two cells of
            // a division after their placement (k_integrate_divided).
            __syncthreads();
            const bool divides = sm.dflag != 0;   // uniform
            if (FUSE == 2 && !divides && i < NODES) d.Xe[g] = x4;
            if (!divides && i < NODES) disp = next_kick(d, P, g, x4, v4, fdk);
            for (int o = 16; o > 0; o >>= 1) disp = fmaxf(disp, __shfl_xor_sync(0xffffffffu, disp, o));
            if ((i & 31) == 0) smax[i >> 5] = disp;
            __syncthreads();
        }
        if (i == 0) {
            if (FUSE && (!DIV || sm.dflag == 0)) {
                float mx = smax[0];  // visible: cell_geom (and the division decision) synchronise the block
                for (int q = 1; q < SLOTS / 32; ++q) mx = fmaxf(mx, smax[q]);
                atomicMax(&st->disp_step, __float_as_uint(mx));
            }
            d.CM[a] = make_float4(cm.x, cm.y, cm.z, 0.f);
            d.aabb[pn][2 * a] = lo;
            d.aabb[pn][2 * a + 1] = hi;
            if (inst != acc_inst) {
                if (acc_inst >= 0) flush_mm(d, acc_inst, pn, acc);
                acc_inst = inst;
                acc[0] = lo.x; acc[1] = hi.x; acc[2] = lo.y; acc[3] = hi.y; acc[4] = lo.z; acc[5] = hi.z;
            } else {
                acc[0] = fminf(acc[0], lo.x); acc[1] = fmaxf(acc[1], hi.x);
                acc[2] = fminf(acc[2], lo.y); acc[3] = fmaxf(acc[3], hi.y);
                acc[4] = fminf(acc[4], lo.z); acc[5] = fmaxf(acc[5], hi.z);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && acc_inst >= 0) flush_mm(d, acc_inst, pn, acc);
}
// Centre of mass, bounding boxes and grid extents only (initialisation,
// src/GPUbounce.cu:739-763).
__global__ void __launch_bounds__(SLOTS) k_geom(Dev d, int par)
{
    __shared__ float4 xs[SLOTS];
    __shared__ GeomScratch gs;
    const int W = n_work(d);
    const int i = threadIdx.x;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = cell_of(d, w);
        const int inst = inst_of(d, a);
        xs[i] = (i < NODES) ? d.X[(size_t)a * SLOTS + i] : make_float4(0, 0, 0, 0);
        __syncthreads();
        float3 cm;
        float4 lo, hi;
        cell_geom(xs, gs, cm, lo, hi);
        if (i == 0) {
            d.CM[a] = make_float4(cm.x, cm.y, cm.z, 0.f);
            d.aabb[par][2 * a] = lo;
            d.aabb[par][2 * a + 1] = hi;
            int *mm = d.st[inst].mm[par];
            atomicMin(&mm[0], f2o(lo.x)); atomicMax(&mm[1], f2o(hi.x));
            atomicMin(&mm[2], f2o(lo.y)); atomicMax(&mm[3], f2o(hi.y));
            atomicMin(&mm[4], f2o(lo.z)); atomicMax(&mm[5], f2o(hi.z));
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Division (src/GPUbounce.cu:1210-1286, src/postscriptinit.cu:148-256).
// D1: one block per instance, dividers in ascending index order, one RANMAR
// normal each (bit-exact float arithmetic of src/RandomVector.h:8-24).
// ---------------------------------------------------------------------------
__device__ void ranmar_dev(InstState *st, float *out, int len)
{
    for (int v = 0; v < len; ++v) {
        float uni = __fsub_rn(st->u[st->i97], st->u[st->j97]);
        if (uni < 0.0f) uni = __fadd_rn(uni, 1.0f);
        st->u[st->i97] = uni;
        if (--st->i97 == 0) st->i97 = 97;
        if (--st->j97 == 0) st->j97 = 97;
        st->rc = __fsub_rn(st->rc, st->rcd);
        if (st->rc < 0.0f) st->rc = __fadd_rn(st->rc, st->rcm);
        uni = __fsub_rn(uni, st->rc);
        if (uni < 0.0f) uni = __fadd_rn(uni, 1.0f);
        out[v] = uni;
    }
}

__device__ void random_vector_dev(InstState *st, float n[3])
{
    float r[2], s;
    do {
        ranmar_dev(st, r, 2);
        r[0] = __fsub_rn(__fmul_rn(2.0f, r[0]), 1.0f);
        r[1] = __fsub_rn(__fmul_rn(2.0f, r[1]), 1.0f);
        s = __fadd_rn(__fmul_rn(r[0], r[0]), __fmul_rn(r[1], r[1]));
    } while (s >= 1.0f);
    float x1 = r[0], x2 = r[1];
    float q = __fsqrt_rn(__fsub_rn(__fsub_rn(1.0f, __fmul_rn(x1, x1)), __fmul_rn(x2, x2)));
    n[0] = __fmul_rn(__fmul_rn(2.0f, x1), q);
    n[1] = __fmul_rn(__fmul_rn(2.0f, x2), q);
    n[2] = __fsub_rn(1.0f, __fmul_rn(2.0f, __fadd_rn(__fmul_rn(x1, x1), __fmul_rn(x2, x2))));
}

__global__ void __launch_bounds__(256) k_div_select(Dev d, int par)
{
    const int k = blockIdx.x;
    if (k >= d.n_inst) return;
    InstState *st = &d.st[k];
    const InstParams &P = d.prm[k];
    if (!(st->step <= P.div_steps && P.growth > 0.0f)) return;
    __shared__ int cnt;
    __shared__ int warp_cnt[8];
    __shared__ int base_slot;
    const int n0 = st->n;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int mine = 0;
    for (int c = threadIdx.x; c < n0; c += blockDim.x) mine += d.divflag[P.base + c] ? 1 : 0;
    mine = warp_sum(mine);
    if ((threadIdx.x & 31) == 0) atomicAdd(&cnt, mine);
    __syncthreads();
    const int total = cnt;
    if (total == 0) return;
    const int room = P.cap - n0;
    const int ndiv = total < room ? total : room;
    if (threadIdx.x == 0) {
        if (total > room) atomicOr(&st->err, CS3D_ERRBIT_CAPACITY);
        base_slot = atomicAdd(d.div_total, ndiv);
        st->div_count = ndiv;
        atomicOr(&d.flags[1], 1);
    }
    __syncthreads();
    // ascending compaction in chunks of blockDim
    int done = 0;
    for (int c0 = 0; c0 < n0 && done < ndiv; c0 += blockDim.x) {
        int c = c0 + threadIdx.x;
        int f = (c < n0) ? (d.divflag[P.base + c] ? 1 : 0) : 0;
        unsigned b = __ballot_sync(0xffffffffu, f);
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) warp_cnt[wid] = __popc(b);
        __syncthreads();
        int off = done;
        for (int q = 0; q < wid; ++q) off += warp_cnt[q];
        off += __popc(b & ((1u << lane) - 1u));
        if (f && off < ndiv) {
            DivEntry &e = d.divtab[base_slot + off];
            e.parent = P.base + c;
            e.daughter = P.base + n0 + off;
            e.inst = k;
        }
        int tot = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) tot += warp_cnt[q];
        done += tot;
        __syncthreads();
    }
    // normals in ascending order (one serial RNG stream per instance)
    if (threadIdx.x == 0) {
        int ev0 = atomicAdd(d.n_events, ndiv);
        for (int q = 0; q < ndiv; ++q) {
            DivEntry &e = d.divtab[base_slot + q];
            float n[3];
            random_vector_dev(st, n);
            e.n[0] = n[0]; e.n[1] = n[1]; e.n[2] = n[2];
            float nn = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            if (fabsf(nn - 1.0f) > 1e-3f) atomicOr(&st->err, CS3D_ERRBIT_BAD_NORMAL);
            if (ev0 + q < d.ev_cap) d.events[ev0 + q] = make_int4(k, st->step, e.parent - P.base, e.daughter - P.base);
            if (!d.single) d.work[atomicAdd(d.work_n, 1)] = e.daughter;
        }
        st->n = n0 + ndiv;
        for (int q = 0; q < 3; ++q) {
            st->mm[par ^ 1][2 * q] = f2o(1.0e30f);
            st->mm[par ^ 1][2 * q + 1] = f2o(-1.0e30f);
        }
    }
    for (int c = threadIdx.x; c < n0; c += blockDim.x) d.divflag[P.base + c] = 0;
}

// D2: one block per division: the two daughters by half-space projection
// through CM + n*gap/2 (FP64 geometry), velocities, pressures, stiffness.
__global__ void __launch_bounds__(SLOTS) k_div_apply(Dev d, int par)
{
    __shared__ float4 xs[SLOTS];
    __shared__ GeomScratch gs;
    const int T = *d.div_total;
    const int pn = par ^ 1;
    const int i = threadIdx.x;
    for (int q = blockIdx.x; q < T; q += gridDim.x) {
        DivEntry e = d.divtab[q];
        const InstParams &P = d.prm[e.inst];
        const int a = e.parent, b = e.daughter;
        float4 cm4 = d.CM[a];
        double half = (double)(0.5f * P.rr);
        double cm[3] = {cm4.x, cm4.y, cm4.z};
        float4 xa = make_float4(0, 0, 0, 0), xb = make_float4(0, 0, 0, 0);
        if (i < NODES) {
            float4 x = d.X[(size_t)a * SLOTS + i];
            double px[3] = {x.x, x.y, x.z};
            // separate roundings (no DFMA) so the result is bit-identical to
            // the oracle's FP64 restatement of CalcAndUpdateDaughtPos
            for (int s = 0; s < 2; ++s) {
                double sg = s == 0 ? 1.0 : -1.0;
                double n[3] = {sg * e.n[0], sg * e.n[1], sg * e.n[2]};
                double o[3], y[3];
                for (int q = 0; q < 3; ++q) {
                    o[q] = __dadd_rn(cm[q], __dmul_rn(half, n[q]));
                    y[q] = __dsub_rn(px[q], o[q]);
                }
                double dn = __dadd_rn(__dadd_rn(__dmul_rn(y[0], n[0]), __dmul_rn(y[1], n[1])), __dmul_rn(y[2], n[2]));
                if (dn <= 0.0)
                    for (int q = 0; q < 3; ++q) y[q] = __dsub_rn(y[q], __dmul_rn(dn, n[q]));
                float4 r = make_float4((float)__dadd_rn(y[0], o[0]), (float)__dadd_rn(y[1], o[1]),
                                       (float)__dadd_rn(y[2], o[2]), 0.f);
                if (s == 0) xa = r; else xb = r;
            }
        }
        __syncthreads();
        xs[i] = xa;
        __syncthreads();
        float3 c1;
        float4 lo, hi;
        cell_geom(xs, gs, c1, lo, hi);
        if (i == 0) { d.aabb[pn][2 * a] = lo; d.aabb[pn][2 * a + 1] = hi; }
        __syncthreads();
        xs[i] = xb;
        __syncthreads();
        cell_geom(xs, gs, c1, lo, hi);
        if (i == 0) {
            d.aabb[pn][2 * b] = lo;
            d.aabb[pn][2 * b + 1] = hi;
            d.press[a] = P.minp;
            d.press[b] = P.minp;
            d.E[b] = P.daught_same ? d.E[a] : P.stiff1;
            d.cell_inst[b] = e.inst;
            d.dirty[a] = 1;  // lists rebuilt around the two cells next step
            d.dirty[b] = 1;
        }
        if (i < NODES) {
            size_t ga = (size_t)a * SLOTS + i, gb = (size_t)b * SLOTS + i;
            d.X[ga] = xa;
            d.X[gb] = xb;
            d.Xb[ga] = xa;   // new anchors of the displacement test
            d.Xb[gb] = xb;
            d.Xe[ga] = xa;   // step-end state of the two cells (read back after a fused last step)
            d.Xe[gb] = xb;
            d.Vb[gb] = d.Vb[ga];
            d.V[gb] = d.V[ga];
            d.FC[gb] = make_float4(0, 0, 0, 0);
            d.FD[gb] = make_float4(0, 0, 0, 0);
        }
        __syncthreads();
    }
}

// CoM correction at the end of a step (correct_com, src/GPUbounce.cu:1430-1440
// with calc_sys_CM :2504-2520 and CorrectCoMMotion, src/propagate.cu:766-776):
// the mean of the cells' centres of mass (a float sum in cell order, as the
// host loop does; a daughter's entry is still 0 in its first step) is
// subtracted from every node.  The centres of mass, boxes and grid of this
// step keep their unshifted values, as in the reference; the list anchors
// move with the nodes (a uniform shift changes no distance).  One block per
// instance.
__global__ void __launch_bounds__(256) k_com_shift(Dev d)
{
    const int k = blockIdx.x;
    if (k >= d.n_inst) return;
    const InstParams &P = d.prm[k];
    if (!P.correct_com) return;
    __shared__ float sys[3];
    const int n = d.st[k].n;
    if (threadIdx.x == 0) {
        float sx = 0.0f, sy = 0.0f, sz = 0.0f;
        for (int c = 0; c < n; ++c) {
            const float4 cm = d.CM[P.base + c];
            sx = __fadd_rn(sx, cm.x);
            sy = __fadd_rn(sy, cm.y);
            sz = __fadd_rn(sz, cm.z);
        }
        sys[0] = __fdiv_rn(sx, (float)n);
        sys[1] = __fdiv_rn(sy, (float)n);
        sys[2] = __fdiv_rn(sz, (float)n);
        d.st[k].syscm[0] = sys[0];
        d.st[k].syscm[1] = sys[1];
        d.st[k].syscm[2] = sys[2];
    }
    __syncthreads();
    const float ox = sys[0], oy = sys[1], oz = sys[2];
    for (int q = threadIdx.x; q < n * SLOTS; q += blockDim.x) {
        const size_t g = (size_t)P.base * SLOTS + q;
        float4 x = d.X[g], b = d.Xb[g];
        x.x = __fsub_rn(x.x, ox); x.y = __fsub_rn(x.y, oy); x.z = __fsub_rn(x.z, oz);
        b.x = __fsub_rn(b.x, ox); b.y = __fsub_rn(b.y, oy); b.z = __fsub_rn(b.z, oz);
        d.X[g] = x;
        d.Xb[g] = b;
    }
}

// calc_sys_CM, src/GPUbounce.cu:2504-2520: the float mean of the first n
// centres of mass, summed in cell order; recorded as the instance's system
// centre.
__device__ float3 sys_centre(const Dev &d, const InstParams &P, InstState *st, int n)
{
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int c = 0; c < n; ++c) {
        const float4 cm = d.CM[P.base + c];
        sx = __fadd_rn(sx, cm.x);
        sy = __fadd_rn(sy, cm.y);
        sz = __fadd_rn(sz, cm.z);
    }
    sx = __fdiv_rn(sx, (float)n);
    sy = __fdiv_rn(sy, (float)n);
    sz = __fdiv_rn(sz, (float)n);
    st->syscm[0] = sx;
    st->syscm[1] = sy;
    st->syscm[2] = sz;
    return make_float3(sx, sy, sz);
}

__device__ __forceinline__ float dist2(float4 cm, float3 o)
{
    const float dx = __fsub_rn(cm.x, o.x), dy = __fsub_rn(cm.y, o.y), dz = __fsub_rn(cm.z, o.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// getRmax2, src/GPUbounce.cu:2523-2536: the largest squared distance of the
// first n centres of mass from the recorded system centre.
__device__ float rmax2_from(const Dev &d, const InstParams &P, const InstState *st, int n)
{
    const float3 o = make_float3(st->syscm[0], st->syscm[1], st->syscm[2]);
    float r2 = 0.0f;
    for (int c = 0; c < n; ++c) {
        const float v = dist2(d.CM[P.base + c], o);
        r2 = r2 < v ? v : r2;   // std::max
    }
    return r2;
}

// num_cells_far, src/GPUbounce.cu:1288-1290 and :2538-2565, after the
// divisions of a step (count_only_internal_cells): the newest div_count cells
// whose centre of mass lies farther than radius_cutoff x the largest distance
// from the system's centre are not counted as dividing.  The daughters'
// centres of mass are still 0 here (computed in their first step), as in the
// reference.  One thread per instance.
__global__ void k_far_count(Dev d)
{
    const int k = blockIdx.x;
    if (k >= d.n_inst || threadIdx.x != 0) return;
    const InstParams &P = d.prm[k];
    InstState *st = &d.st[k];
    if (!(P.far_r > 0.0f) || !(st->step <= P.div_steps && P.growth > 0.0f)) return;
    const int n = st->n, nd = st->div_count;
    if (nd == 0 || n < 50) return;
    const float3 o = sys_centre(d, P, st, n);
    const float thr = __fmul_rn(__fmul_rn(P.far_r, P.far_r), rmax2_from(d, P, st, n));
    int far = 0;
    for (int c = n - nd; c < n; ++c)
        if (dist2(d.CM[P.base + c], o) > thr) ++far;
    if (far) {
        const int q = atomicAdd(d.n_far, 1);
        if (q < d.far_cap) d.farlog[q] = make_int4(k, st->step, far, 0);
    }
}

// Cells softened when growth ends, src/GPUbounce.cu:1340-1429 (duringGrowth
// off): at the end of step div_time_steps + 2, after the step's grid and
// before its CoM correction.  One thread per instance runs the reference's
// host loops in their order.
__global__ void k_soften(Dev d, int step)
{
    const int k = blockIdx.x;
    if (k >= d.n_inst || threadIdx.x != 0) return;
    const InstParams &P = d.prm[k];
    InstState *st = &d.st[k];
    if (!P.soften || st->step != step || P.div_steps + 2 != step) return;
    const int n = st->n;
    int count = P.soft_n;
    if (P.soft_frac > 0.0f) count = (int)roundf(__fmul_rn(P.soft_frac, (float)n));
    float *E = d.E + P.base;
    if (P.soft_rand) {
        // distinct picks roundf(u * n) in [0, n]; n itself names no cell
        if (count > n + 1) { atomicOr(&st->err, CS3D_ERRBIT_SOFT_CELLS); return; }
        uint8_t *pick = d.pick + P.base + k;
        for (int c = 0; c <= n; ++c) pick[c] = 0;
        long long draws = 0;
        for (int got = 0; got < count;) {
            if (++draws > 64ll * (n + 1) + (1ll << 20)) { atomicOr(&st->err, CS3D_ERRBIT_SOFT_CELLS); break; }
            float u;
            ranmar_dev(st, &u, 1);
            const int ind = (int)roundf(__fmul_rn(u, (float)n));
            if (!pick[ind]) { pick[ind] = 1; ++got; }
        }
        for (int c = 0; c < n; ++c)
            if (pick[c]) E[c] = P.E2;
        return;
    }
    // getRmax2 runs before calc_sys_CM here (src/GPUbounce.cu:1399-1402), so
    // it measures from the previously recorded system centre
    const float r2max = rmax2_from(d, P, st, n);
    const float3 o = sys_centre(d, P, st, n);
    const float f = __fsub_rn(1.0f, P.closeness);
    const float thr = __fmul_rn(__fmul_rn(f, f), r2max);
    for (int c = 0, got = 0; got < count && c < n; ++c)
        if (dist2(d.CM[P.base + c], o) <= thr) { E[c] = P.E2; ++got; }
}

// Volume histogram of one instance's cells at the current positions (the
// analysis scripts/pop.py and the statistical checks do offline): one block
// per cell computes the centre of mass and the volume of src/volume.cu:5-163
// in FP64 (the division test's arithmetic) and counts it into one of nbins
// equal bins over [lo, hi), counts[0] below, counts[nbins + 1] at or above.
__global__ void __launch_bounds__(SLOTS) k_vol_hist(Dev d, int inst, float lo, float hi, int nbins,
                                                    unsigned long long *counts, float *vols)
{
    __shared__ float4 xs[SLOTS];
    __shared__ GeomScratch gs;
    const InstParams &P = d.prm[inst];
    const int n = d.st[inst].n;
    for (int c = blockIdx.x; c < n; c += gridDim.x) {
        const int a = P.base + c;
        const int i = threadIdx.x;
        xs[i] = i < NODES ? d.X[(size_t)a * SLOTS + i] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        float3 cm;
        float4 blo, bhi;
        cell_geom(xs, gs, cm, blo, bhi);
        double vol, area;
        cell_volume(d, xs, cm, gs, false, vol, area);
        if (i == 0) {
            const float v = (float)vol;
            if (vols) vols[c] = v;
            int b;
            if (!(v >= lo)) b = 0;
            else if (!(v < hi)) b = nbins + 1;
            else {
                b = 1 + (int)((double)(v - lo) / ((double)hi - (double)lo) * nbins);
                b = b > nbins ? nbins : b;
            }
            atomicAdd(&counts[b], 1ull);
        }
        __syncthreads();
    }
}

// G: grid extents of instances that divided this step, from all boxes.
__global__ void k_grid_fix(Dev d, int par)
{
    const int pn = par ^ 1;
    const int W = n_work(d);
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        int a = cell_of(d, w);
        int inst = inst_of(d, a);
        if (d.st[inst].div_count == 0) continue;
        float4 lo = d.aabb[pn][2 * a], hi = d.aabb[pn][2 * a + 1];
        int *mm = d.st[inst].mm[pn];
        atomicMin(&mm[0], f2o(lo.x)); atomicMax(&mm[1], f2o(hi.x));
        atomicMin(&mm[2], f2o(lo.y)); atomicMax(&mm[3], f2o(hi.y));
        atomicMin(&mm[4], f2o(lo.z)); atomicMax(&mm[5], f2o(hi.z));
    }
}

// ---------------------------------------------------------------------------
// Neighbour-list build (instances whose displacement bound reached the skin,
// or that divided).  The nodes are binned in cubes of edge hb slightly above
// the list radius and the bins hashed into the instance's slice of the
// buckets; a counting sort puts the positions in bucket order (hpos).
// Bucket of bin (ix, iy, iz): the low bits of each coordinate side by side,
// so that the 27 bins around a node fall in 27 distinct buckets and the three
// bins along x are (unless they wrap) three consecutive buckets.
// ---------------------------------------------------------------------------
struct BinGeom {
    float inv;          // 1 / bin edge
    int bx, by;         // bits of x, y in the bucket number
    unsigned mask;      // slice size - 1
    unsigned base;      // first bucket of the instance's slice
};

__device__ __forceinline__ BinGeom bin_geom(const Dev &d, int inst)
{
    const InstState &st = d.st[inst];
    BinGeom b;
    // bin edge 1% above the list radius: float rounding of x / edge cannot
    // put two nodes closer than the radius more than one bin apart
    b.inv = 1.0f / ((st.rcur + 1e-4f) * 1.01f);
    const int B = st.hbits;
    b.bx = B / 3;
    b.by = B / 3;
    b.mask = (1u << B) - 1u;
    b.base = st.hbase;
    return b;
}

__device__ __forceinline__ int bin_coord(float v, float inv)
{
    return (int)floorf(fminf(fmaxf(v * inv, -1.0e9f), 1.0e9f));
}

constexpr int CB = 4;  // hash candidates loaded together in the list build

__device__ __forceinline__ unsigned bucket_of(const BinGeom &b, int ix, int iy, int iz)
{
    const unsigned code = ((unsigned)ix & ((1u << b.bx) - 1u)) | (((unsigned)iy & ((1u << b.by) - 1u)) << b.bx) |
                          ((unsigned)iz << (b.bx + b.by));
    return b.base + (code & b.mask);
}

// B1: zero the bucket counts (hsize + SCAN_TILE entries, the tail pads the
// last scan tile).
__global__ void k_nh_zero(Dev d)
{
    if (!d.flags[0]) return;
    int4 *p = reinterpret_cast<int4 *>(d.hcount);
    const int n4 = (*d.hsz + SCAN_TILE) / 4;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += gridDim.x * blockDim.x)
        p[q] = make_int4(0, 0, 0, 0);
}

// B2: count the nodes of every bucket; each node keeps its rank.
__global__ void __launch_bounds__(SLOTS) k_nh_count(Dev d)
{
    if (!d.flags[0]) return;
    const int W = n_work(d);
    const int i = threadIdx.x;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = cell_of(d, w);
        const int inst = inst_of(d, a);
        if (!d.st[inst].rebuild || i >= NODES) continue;
        const BinGeom b = bin_geom(d, inst);
        const size_t g = (size_t)a * SLOTS + i;
        const float4 x = d.X[g];
        const unsigned k = bucket_of(b, bin_coord(x.x, b.inv), bin_coord(x.y, b.inv), bin_coord(x.z, b.inv));
        d.node_rank[g] = atomicAdd(&d.hcount[k], 1);
    }
}

// B3: sums of the scan tiles.
__global__ void __launch_bounds__(256) k_nh_scan_tiles(Dev d)
{
    if (!d.flags[0]) return;
    __shared__ int wsum[32];
    const int ntile = *d.hsz / SCAN_TILE + 1;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
        const int4 *p = reinterpret_cast<const int4 *>(d.hcount + (size_t)t * SCAN_TILE);
        int s = 0;
#pragma unroll
        for (int q = 0; q < SCAN_TILE / 4 / 256; ++q) {
            const int4 v = p[threadIdx.x + q * 256];
            s += v.x + v.y + v.z + v.w;
        }
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int q = 0; q < 8; ++q) tot += wsum[q];
            d.hscan[t] = tot;
        }
        __syncthreads();
    }
}

// B4: exclusive scan of the tile sums (one block).
__global__ void __launch_bounds__(1024) k_nh_scan_top(Dev d)
{
    if (!d.flags[0]) return;
    __shared__ int wsum[32];
    __shared__ int carry;
    const int ntile = *d.hsz / SCAN_TILE + 1;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int t0 = 0; t0 < ntile; t0 += 1024) {
        const int t = t0 + threadIdx.x;
        const int v = t < ntile ? d.hscan[t] : 0;
        int tot;
        const int e = block_excl_scan<1024>(v, wsum, tot);
        if (t < ntile) d.hscan[t] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

// B5: bucket starts (exclusive scan of the counts, in place).
__global__ void __launch_bounds__(256) k_nh_scan_apply(Dev d)
{
    if (!d.flags[0]) return;
    __shared__ int wsum[32];
    constexpr int PER = SCAN_TILE / 256;  // 16 consecutive buckets per thread
    const int ntile = *d.hsz / SCAN_TILE + 1;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
        int4 *p = reinterpret_cast<int4 *>(d.hcount + (size_t)t * SCAN_TILE + threadIdx.x * PER);
        int4 v[PER / 4];
        int s = 0;
#pragma unroll
        for (int q = 0; q < PER / 4; ++q) {
            v[q] = p[q];
            s += v[q].x + v[q].y + v[q].z + v[q].w;
        }
        int tot;
        int run = d.hscan[t] + block_excl_scan<256>(s, wsum, tot);
#pragma unroll
        for (int q = 0; q < PER / 4; ++q) {
            int4 o;
            o.x = run; run += v[q].x;
            o.y = run; run += v[q].y;
            o.z = run; run += v[q].z;
            o.w = run; run += v[q].w;
            p[q] = o;
        }
    }
}

// B6: positions in bucket order.
__global__ void __launch_bounds__(SLOTS) k_nh_fill(Dev d)
{
    if (!d.flags[0]) return;
    const int W = n_work(d);
    const int i = threadIdx.x;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = cell_of(d, w);
        const int inst = inst_of(d, a);
        if (!d.st[inst].rebuild || i >= NODES) continue;
        const BinGeom b = bin_geom(d, inst);
        const size_t g = (size_t)a * SLOTS + i;
        const float4 x = d.X[g];
        const unsigned k = bucket_of(b, bin_coord(x.x, b.inv), bin_coord(x.y, b.inv), bin_coord(x.z, b.inv));
        // w: the node as cell << 8 | node (cells < 2^23)
        d.hpos[d.hcount[k] + d.node_rank[g]] = make_float4(x.x, x.y, x.z, __int_as_float((a << 8) | i));
    }
}

// B7: per cell, from the nodes of other cells within the list radius of its
// nodes: the candidate cells (ascending id) and each node's entries
// (slot << 8 | node, ascending: by candidate cell, then node).  Candidate
// cells are first collected in a shared open-addressing set ("temporary
// slots"), each node's entries kept as (temporary slot, node) and remapped
// once the slots are sorted.
struct BuildSmem {
    int tkey[256];           // candidate cell of each temporary slot, -1 if free
    uint32_t mask[256][6];   // partner nodes of each temporary slot (CS3D_OPT_HALO_STATS)
    int comp_key[256], comp_t[256];
    short slot_of_t[256];    // final slot of a temporary slot, -1 if dropped
    int slot_t[MAXC];        // temporary slot of each final slot
    int wsum[32];
    int ncomp;
    int flag;
};

// Phase 0 builds the cells of whole-instance rebuilds and the divided cells
// (dirty 1) of partial ones, and marks the candidates of the divided cells
// (dirty 2); phase 1 builds the marked cells and clears all marks.
__global__ void __launch_bounds__(SLOTS) k_nl_cell(Dev d, int phase)
{
    if (!d.flags[0]) return;
    __shared__ BuildSmem sm;
    const int W = n_work(d);
    const int i = threadIdx.x;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = cell_of(d, w);
        const int inst = inst_of(d, a);
        InstState *st = &d.st[inst];
        const int rb = st->rebuild;
        if (!rb) continue;  // uniform across the block
        __syncthreads();
        if (i == 0) sm.flag = d.dirty[a];
        __syncthreads();
        const int mark = sm.flag;
        if (phase == 1 && mark && i == 0) d.dirty[a] = 0;
        const bool build = phase == 0 ? (rb == 2 || mark == 1) : (rb == 1 && mark == 2);
        if (!build) continue;
        const BinGeom b = bin_geom(d, inst);
        const float rl = st->rcur + 1e-4f;
        const float rl2 = rl * rl;
        const bool halo = d.halo_stats != 0;   // uniform
        for (int t = i; t < 256; t += SLOTS) sm.tkey[t] = -1;
        if (halo)
            for (int q = i; q < 256 * 6; q += SLOTS) (&sm.mask[0][0])[q] = 0u;
        if (i == 0) sm.ncomp = 0;
        __syncthreads();
        const size_t g = (size_t)a * SLOTS + i;
        const float4 x = (i < NODES) ? d.X[g] : make_float4(0, 0, 0, 0);
        uint16_t *ep = d.ent + (size_t)a * MAXE * SLOTS + i;
        int cnt = 0;
        bool lost = false;
        if (i < NODES) {
            const int ix = bin_coord(x.x, b.inv), iy = bin_coord(x.y, b.inv), iz = bin_coord(x.z, b.inv);
            int last_c = -1, last_t = -1;
            for (int r = 0; r < 9; ++r) {
                const int jy = iy + (r % 3) - 1, jz = iz + r / 3 - 1;
                const unsigned k0 = bucket_of(b, ix - 1, jy, jz);
                const unsigned k2 = bucket_of(b, ix + 1, jy, jz);
                // three consecutive buckets unless the x bits or the table wrap
                const int nrun = (k2 == k0 + 2u) ? 1 : 3;
                for (int u = 0; u < nrun; ++u) {
                    unsigned kb, ke;
                    if (nrun == 1) { kb = k0; ke = k0 + 3u; }
                    else { kb = bucket_of(b, ix - 1 + u, jy, jz); ke = kb + 1u; }
                    const int p0 = d.hcount[kb], p1 = d.hcount[ke];
                    // candidates in batches: the loads of a batch are in flight together;
                    // past the run a far sentinel fails the distance test
                    for (int p = p0; p < p1; p += CB) {
                      float4 yb[CB];
#pragma unroll
                      for (int q = 0; q < CB; ++q)
                          yb[q] = p + q < p1 ? d.hpos[p + q] : make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.f);
#pragma unroll
                      for (int q = 0; q < CB; ++q) {
                        const float4 y = yb[q];
                        // the distance first: most candidates fail it
                        const float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
                        if (!(dx * dx + dy * dy + dz * dz < rl2)) continue;
                        // the instance's own hash slice holds only its own nodes
                        const int id = __float_as_int(y.w);
                        const int c = id >> 8;
                        if (c == a) continue;
                        int t = last_t;
                        if (c != last_c) {
                            t = -1;
                            unsigned q = ((unsigned)c * 2654435761u) >> 24;
                            for (int probe = 0; probe < 256; ++probe, q = (q + 1u) & 255u) {
                                const int old = atomicCAS(&sm.tkey[q], -1, c);
                                if (old == -1 || old == c) { t = (int)q; break; }
                            }
                            if (t < 0) { lost = true; continue; }
                            last_c = c;
                            last_t = t;
                        }
                        const int j = id & 255;
                        if (halo) atomicOr(&sm.mask[t][j >> 5], 1u << (j & 31));
                        if (cnt < MAXE) ep[(size_t)cnt * SLOTS] = (uint16_t)((t << 8) | j);
                        ++cnt;
                      }
                    }
                }
            }
        }
        __syncthreads();
        for (int t = i; t < 256; t += SLOTS) {
            const int c = sm.tkey[t];
            if (c >= 0) {
                const int q = atomicAdd(&sm.ncomp, 1);
                sm.comp_key[q] = c;
                sm.comp_t[q] = t;
            }
        }
        __syncthreads();
        const int nct = sm.ncomp;
        for (int q = i; q < nct; q += SLOTS) {
            const int key = sm.comp_key[q];
            int r = 0;
            for (int m = 0; m < nct; ++m) r += sm.comp_key[m] < key;
            const int t = sm.comp_t[q];
            sm.slot_of_t[t] = (short)(r < MAXC ? r : -1);
            if (r < MAXC) {
                sm.slot_t[r] = t;
                d.cand[(size_t)a * MAXC + r] = key;
            }
        }
        __syncthreads();
        const int nc = nct < MAXC ? nct : MAXC;
        // distinct partner nodes of the cell (statistics, CS3D_OPT_HALO_STATS)
        int nh = 0;
        if (halo) {
            int ns = 0;
            if (i < nc) {
                const int t = sm.slot_t[i];
#pragma unroll
                for (int k = 0; k < 6; ++k) ns += __popc(sm.mask[t][k]);
            }
            block_excl_scan<SLOTS>(ns, sm.wsum, nh);
        }
        // entries: (temporary slot, node) -> (slot, node), ascending
        if (i < NODES) {
            uint16_t ord[MAXE];
            int m = 0;
            const int ne = cnt < MAXE ? cnt : MAXE;
            for (int k = 0; k < ne; ++k) {
                const unsigned e = ep[(size_t)k * SLOTS];
                const int s = sm.slot_of_t[e >> 8];
                if (s < 0) continue;
                const unsigned h = ((unsigned)s << 8) | (e & 255u);
                int pos = m;
                while (pos > 0 && ord[pos - 1] > h) { ord[pos] = ord[pos - 1]; --pos; }
                ord[pos] = (uint16_t)h;
                ++m;
            }
            for (int k = 0; k < m; ++k) ep[(size_t)k * SLOTS] = ord[k];
            d.nent[g] = (uint8_t)m;
            // new anchors, except for the neighbours of divided cells: other
            // cells' lists rely on their old anchors
            if (phase == 0) d.Xb[g] = x;
            if (cnt > MAXE) atomicOr(&st->err, CS3D_ERRBIT_ENTRY_OVERFLOW);
            if (lost) atomicOr(&st->err, CS3D_ERRBIT_CAND_OVERFLOW);
        } else {
            d.nent[g] = 0;
        }
        if (phase == 0 && rb == 1 && i < nc) atomicCAS(&d.dirty[d.cand[(size_t)a * MAXC + i]], 0, 2);
        if (i == 0) {
            if (nct > MAXC) atomicOr(&st->err, CS3D_ERRBIT_CAND_OVERFLOW);
            atomicAdd(&st->built, 1);
            d.ncand[a] = nc;
            atomicMax(&st->max_cand, nct);
            if (halo) atomicMax(&st->max_halo, nh);
        }
        int wm = cnt;
        for (int o = 16; o > 0; o >>= 1) wm = max(wm, __shfl_xor_sync(0xffffffffu, wm, o));
        if ((i & 31) == 0) atomicMax(&st->max_entries, wm);
        __syncthreads();
    }
}

}  // namespace cs3d
