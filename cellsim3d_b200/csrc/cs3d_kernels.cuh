// cs3d_kernels.cuh -- the per-timestep kernels of libcs3d.so (sm_100a).
//
// One CTA of 192 threads (six warps) owns one cell at a time and walks the
// active-cell work table grid-stride; thread i owns node i.  The cell's 180
// positions and velocities are staged in shared memory; the 540 bond angles
// are evaluated once each (the reference evaluates each twice, once from the
// vertex and once from the arm end) and their arm-end forces are gathered
// from shared memory in the reference's summation order.  Inter-cell contact
// candidates come from a per-node neighbour list built on the device and
// reused while the accumulated displacement stays inside the skin; the exact
// reference predicates (stale bounding box, stale grid bin, strict and
// non-strict cut-offs) are re-evaluated on every candidate every step, so the
// pair sets are exactly the reference's.
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

// Kick of the split velocity Verlet with the reference's mixed precision:
// the float sum is scaled by the double literal 0.5 and divided by the mass
// in double, then stored as float (src/propagate.cu:698-705, 721-723, 732-734).
__device__ __forceinline__ float kick(float v, float fsum, double m)
{
    return (float)((double)v + 0.5 * (double)fsum / m);
}

// Bond-angle term for one angle at a vertex with arms P (to the p-end node)
// and Q (to the q-end node); Fp/Fq are GetAngleForce(P, Q) and
// GetAngleForce(Q, P) of src/propagate.cu:26-60 (k = 1000, :335).
__device__ __forceinline__ void angle_pair(float3 P, float3 Q, float th0, float3 &Fp, float3 &Fq)
{
#ifdef CS3D_ANGLE_F64
    double px = P.x, py = P.y, pz = P.z, qx = Q.x, qy = Q.y, qz = Q.z;
    double idk = px * qx + py * qy + pz * qz;
    double rp2 = px * px + py * py + pz * pz;
    double rq2 = qx * qx + qy * qy + qz * qz;
    double c1 = -1.0 / sqrt(rp2 * rq2 - idk * idk + 1e-3);
    double th = acos(idk / (sqrt(rp2) * sqrt(rq2) + 1e-3));
    double f = -1000.0 * c1 * (th - (double)th0);
    double cp = idk / rp2, cq = idk / rq2;
    Fp = make_float3((float)(f * (qx - cp * px)), (float)(f * (qy - cp * py)), (float)(f * (qz - cp * pz)));
    Fq = make_float3((float)(f * (px - cq * qx)), (float)(f * (py - cq * qy)), (float)(f * (pz - cq * qz)));
#else
    float idk = dot3(P, Q);
    float rp2 = dot3(P, P);
    float rq2 = dot3(Q, Q);
    float c1 = -1.0f / sqrtf((float)((double)(rp2 * rq2 - idk * idk) + 1e-3));
    float th = (float)acos((double)idk / ((double)(sqrtf(rp2) * sqrtf(rq2)) + 1e-3));
    float f = -1000.0f * c1 * (th - th0);
    float cp = idk / rp2, cq = idk / rq2;
    Fp = make_float3(f * (Q.x - cp * P.x), f * (Q.y - cp * P.y), f * (Q.z - cp * P.z));
    Fq = make_float3(f * (P.x - cq * Q.x), f * (P.y - cq * Q.y), f * (P.z - cq * Q.z));
#endif
}

// Shared per-CTA data of the contact sweep: the candidate cells of the
// current cell with their stale boxes and stale insertion bin ranges.
struct SlotData {
    int cell[MAXC];
    float4 lo[MAXC], hi[MAXC];
    int rlo[MAXC][3], rhi[MAXC][3];
    int ncand;
    float mn[3];
    int div[3];
};

// Fill SlotData for cell a (threads 0..MAXC-1).  Must be followed by a
// __syncthreads().
__device__ __forceinline__ void load_slots(const Dev &d, int a, const InstParams &P, const InstState *st,
                                           int par, SlotData &sd)
{
    int t = threadIdx.x;
    int nc = d.ncand[a];
    if (t == 0) {
        sd.ncand = nc;
        const int *mm = st->mm[par];
        for (int q = 0; q < 3; ++q) {
            float mn = fminf(o2f(mm[2 * q]), 1.0e8f);
            float mx = fmaxf(o2f(mm[2 * q + 1]), -1.0e8f);
            sd.mn[q] = mn;
            sd.div[q] = grid_div(mn, mx);
        }
    }
    __syncthreads();
    if (t < nc) {
        int c = d.cand[a * MAXC + t];
        sd.cell[t] = c;
        float4 lo = d.aabb[par][2 * c], hi = d.aabb[par][2 * c + 1];
        sd.lo[t] = lo;
        sd.hi[t] = hi;
        bin_range_axis(lo.x, hi.x, P.ra, sd.mn[0], sd.div[0], sd.rlo[t][0], sd.rhi[t][0]);
        bin_range_axis(lo.y, hi.y, P.ra, sd.mn[1], sd.div[1], sd.rlo[t][1], sd.rhi[t][1]);
        bin_range_axis(lo.z, hi.z, P.ra, sd.mn[2], sd.div[2], sd.rlo[t][2], sd.rhi[t][2]);
    }
}

// ---------------------------------------------------------------------------
// Contact sweep of one node over its neighbour-list entries.
// MODE 0: conservative + dissipative (S1); MODE 1: dissipative only (S2).
// ---------------------------------------------------------------------------
template <int MODE>
__device__ __forceinline__ void contact_sweep(const Dev &d, const InstParams &P, const SlotData &sd,
                                              int a, int i, float3 x, float3 v, float3 nrm,
                                              const float4 *__restrict__ Vsrc, float3 &cf, float3 &vt)
{
    int nb[3] = {node_bin_axis(x.x, sd.mn[0], sd.div[0]), node_bin_axis(x.y, sd.mn[1], sd.div[1]),
                 node_bin_axis(x.z, sd.mn[2], sd.div[2])};
    int ne = d.nent[a * SLOTS + i];
    int cur = -1;
    bool ok = false;
    int c = 0;
    for (int k = 0; k < ne; ++k) {
        unsigned e = d.ent[((size_t)a * MAXE + k) * SLOTS + i];
        int s = (int)(e >> 8), j = (int)(e & 255u);
        if (s != cur) {
            cur = s;
            c = sd.cell[s];
            ok = nb[0] >= sd.rlo[s][0] && nb[0] <= sd.rhi[s][0] && nb[1] >= sd.rlo[s][1] &&
                 nb[1] <= sd.rhi[s][1] && nb[2] >= sd.rlo[s][2] && nb[2] <= sd.rhi[s][2] &&
                 aabb_keep(sd.lo[s], sd.hi[s], x.x, x.y, x.z, P.ra2);
        }
        if (!ok) continue;
        size_t gj = (size_t)c * SLOTS + j;
        float4 xj = __ldg(&d.X[gj]);
        float dx = __fsub_rn(x.x, xj.x), dy = __fsub_rn(x.y, xj.y), dz = __fsub_rn(x.z, xj.z);
        float r2 = r2_nc(dx, dy, dz);
        if (r2 > P.ra2) continue;
        // dissipative pair (non-strict cut-off, src/propagate.cu:641)
        float4 vj = __ldg(&Vsrc[gj]);
        float3 vij = make_float3(v.x - vj.x, v.y - vj.y, v.z - vj.z);
        float dn = dot3(vij, nrm);
        vt.x += vij.x - dn * nrm.x;
        vt.y += vij.y - dn * nrm.y;
        vt.z += vij.z - dn * nrm.z;
        if (MODE == 0) {
            if (d.record_pairs) {
                unsigned long long slot = atomicAdd(d.n_pairs, 1ull);
                if ((long long)slot < d.pair_cap)
                    d.pairs[slot] = make_int4((a << 8) | i, (c << 8) | j, r2 < P.ra2 ? 3 : 2, 0);
            }
            if (r2 < P.ra2) {  // conservative pair (strict cut-off, src/propagate.cu:421)
                float R = sqrtf(r2);
                float k = 0.0f;
                if (R < P.ra) k += -P.asE * (P.ra - R) / R;
                if (R <= P.rr) k += P.rsE * (P.rr - R) / R;
                cf.x += k * dx;
                cf.y += k * dy;
                cf.z += k * dz;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// K1: first half kick + drift of a step (Integrate + ForwardTime,
// src/propagate.cu:681-763) and PressureUpdate (src/PressureKernels.cu:35-39).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SLOTS) k_integrate(Dev d)
{
    const int W = *d.work_n;
    __shared__ float smax[SLOTS / 32];
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        int a = d.work[w];
        int inst = d.cell_inst[a];
        const InstParams &P = d.prm[inst];
        int i = threadIdx.x;
        float disp = 0.0f;
        if (i < NODES) {
            size_t g = (size_t)a * SLOTS + i;
            float4 x = d.X[g], v = d.V[g], fc = d.FC[g], fd = d.FD[g];
            const float dt = P.dt;
            const double m = P.mass;
            v.x = kick(v.x, __fadd_rn(__fmul_rn(dt, fc.x), __fmul_rn(dt, fd.x)), m);
            v.y = kick(v.y, __fadd_rn(__fmul_rn(dt, fc.y), __fmul_rn(dt, fd.y)), m);
            v.z = kick(v.z, __fadd_rn(__fmul_rn(dt, fc.z), __fmul_rn(dt, fd.z)), m);
            float4 xn = make_float4(__fmaf_rn(v.x, dt, x.x), __fmaf_rn(v.y, dt, x.y), __fmaf_rn(v.z, dt, x.z), 0.0f);
            float ddx = xn.x - x.x, ddy = xn.y - x.y, ddz = xn.z - x.z;
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
            if (d.press[a] < P.maxp) d.press[a] = d.press[a] + P.growth;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Per-step bookkeeping (one block): step counter, rebuild decision, reset of
// the accumulators that this step fills.
// ---------------------------------------------------------------------------
__global__ void k_step_begin(Dev d, int par_next)
{
    __shared__ int any;
    if (threadIdx.x == 0) { any = 0; *d.div_total = 0; }
    __syncthreads();
    for (int k = threadIdx.x; k < d.n_inst; k += blockDim.x) {
        InstState *st = &d.st[k];
        const InstParams &P = d.prm[k];
        st->step += 1;
        float ds = __uint_as_float(st->disp_step);
        st->disp_step = 0u;
        // every node moved at most ds this step, so no pair distance changed
        // by more than 2*ds; a margin of 1e-3 covers float rounding
        float acc = st->disp_acc + ds * 1.0001f + 1e-6f;
        bool need = st->force_rebuild || 2.0f * acc + 1e-3f >= P.skin;
        st->rebuild = need ? 1 : 0;
        st->force_rebuild = 0;
        st->disp_acc = need ? 0.0f : acc;
        st->div_count = 0;
        if (need) st->rebuilds += 1;
        for (int q = 0; q < 3; ++q) {
            st->mm[par_next][2 * q] = f2o(1.0e30f);
            st->mm[par_next][2 * q + 1] = f2o(-1.0e30f);
            st->bmm[2 * q] = f2o(1.0e30f);
            st->bmm[2 * q + 1] = f2o(-1.0e30f);
        }
        st->maxext = 0u;
        if (need) any = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) { d.flags[0] = any; *d.n_pairs = 0ull; }
}

// Init variant: rebuild everything, reset parity-0 grid accumulators.
__global__ void k_init_begin(Dev d)
{
    for (int k = threadIdx.x; k < d.n_inst; k += blockDim.x) {
        InstState *st = &d.st[k];
        st->rebuild = 1;
        st->force_rebuild = 0;
        st->disp_acc = 0.0f;
        st->disp_step = 0u;
        for (int p = 0; p < 2; ++p)
            for (int q = 0; q < 3; ++q) {
                st->mm[p][2 * q] = f2o(1.0e30f);
                st->mm[p][2 * q + 1] = f2o(-1.0e30f);
            }
        for (int q = 0; q < 3; ++q) {
            st->bmm[2 * q] = f2o(1.0e30f);
            st->bmm[2 * q + 1] = f2o(-1.0e30f);
        }
        st->maxext = 0u;
    }
    if (threadIdx.x == 0) { d.flags[0] = 1; *d.div_total = 0; *d.n_pairs = 0ull; }
}

// ---------------------------------------------------------------------------
// Block reductions over the 180 nodes of a cell.
// ---------------------------------------------------------------------------
struct GeomScratch {
    double sum[SLOTS / 32][3];
    float mn[SLOTS / 32][3], mx[SLOTS / 32][3];
    double vol[SLOTS / 32], area[SLOTS / 32];
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

// Volume, area and the division test, src/volume.cu:5-163, in FP64.
__device__ __forceinline__ void cell_volume(const Dev &d, const float4 *xs, float3 cm, GeomScratch &gs,
                                            bool sph, double &vol, double &area)
{
    int t = threadIdx.x, w = t >> 5, l = t & 31;
    double tv = 0, fa = 0;
    if (t < CS3D_FACES) {
        const uint8_t *F = d.topo.faces + 7 * t;
        double lx[7], ly[7], lz[7];
        for (int q = 0; q < 7; ++q) {
            float4 p = xs[F[q]];
            lx[q] = (double)p.x - (double)cm.x;
            ly[q] = (double)p.y - (double)cm.y;
            lz[q] = (double)p.z - (double)cm.z;
        }
        double ax = 0, ay = 0, az = 0;
        for (int q = 0; q < 5; ++q) { ax += lx[q]; ay += ly[q]; az += lz[q]; }
        double fac = (double)0.166666667f;
        if (t < 12) fac = (double)0.2f;
        else { ax += lx[5]; ay += ly[5]; az += lz[5]; }
        ax *= fac; ay *= fac; az *= fac;
        for (int q = 0; q < 6; ++q) {
            double n1 = (ly[q + 1] * az - ay * lz[q + 1]) * lx[q];
            double n2 = (lz[q + 1] * ax - az * lx[q + 1]) * ly[q];
            double n3 = (lx[q + 1] * ay - ax * ly[q + 1]) * lz[q];
            tv += fabs(n1 + n2 + n3);
            if (sph) {
                double x1 = lx[q] - ax, y1 = ly[q] - ay, z1 = lz[q] - az;
                double x2 = lx[q + 1] - ax, y2 = ly[q + 1] - ay, z2 = lz[q + 1] - az;
                double xx = y1 * z2 - z1 * y2, yy = z1 * x2 - x1 * z2, zz = x1 * y2 - y1 * x2;
                fa += 0.5 * sqrt(xx * xx + yy * yy + zz * zz);
            }
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
struct S1Smem {
    float4 xs[SLOTS];
    float4 vs[SLOTS];
    float armx[NARM], army[NARM], armz[NARM];
    SlotData sd;
};

template <bool INIT>
__global__ void __launch_bounds__(SLOTS) k_s1(Dev d, int par)
{
    __shared__ S1Smem sm;
    const int W = *d.work_n;
    const int i = threadIdx.x;
    const uint32_t nnp = (i < NODES) ? __ldg(&d.topo.nnpack[i]) : 0u;
    const int n0 = nnp & 255, n1 = (nnp >> 8) & 255, n2 = (nnp >> 16) & 255;
    const float sgn = (float)(int8_t)(nnp >> 24);
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = d.work[w];
        const int inst = d.cell_inst[a];
        const InstParams &P = d.prm[inst];
        const size_t g = (size_t)a * SLOTS + i;
        float4 x4 = make_float4(0, 0, 0, 0), v4 = make_float4(0, 0, 0, 0);
        if (i < NODES) { x4 = d.X[g]; v4 = d.V[g]; }
        sm.xs[i] = x4;
        sm.vs[i] = v4;
        load_slots(d, a, P, &d.st[inst], par, sm.sd);
        __syncthreads();
        const float3 x = f3(x4);
        const float3 v = f3(v4);
        // bond angles: thread = vertex, three angles each
        if (P.angles && i < NODES) {
            float3 pa = sub3(f3(sm.xs[n0]), x), pb = sub3(f3(sm.xs[n1]), x), pc = sub3(f3(sm.xs[n2]), x);
            float4 th = __ldg(&d.topo.th0[i]);
            float3 Fp, Fq;
            angle_pair(pa, pb, th.x, Fp, Fq);
            int o = i * 6;
            sm.armx[o] = Fp.x; sm.army[o] = Fp.y; sm.armz[o] = Fp.z;
            sm.armx[o + 1] = Fq.x; sm.army[o + 1] = Fq.y; sm.armz[o + 1] = Fq.z;
            angle_pair(pb, pc, th.y, Fp, Fq);
            sm.armx[o + 2] = Fp.x; sm.army[o + 2] = Fp.y; sm.armz[o + 2] = Fp.z;
            sm.armx[o + 3] = Fq.x; sm.army[o + 3] = Fq.y; sm.armz[o + 3] = Fq.z;
            angle_pair(pa, pc, th.z, Fp, Fq);
            sm.armx[o + 4] = Fp.x; sm.army[o + 4] = Fp.y; sm.armz[o + 4] = Fp.z;
            sm.armx[o + 5] = Fq.x; sm.army[o + 5] = Fq.y; sm.armz[o + 5] = Fq.z;
        }
        __syncthreads();
        if (i < NODES) {
            if (isnan(x.x) || isnan(x.y) || isnan(x.z)) atomic_or_err(&d.st[inst], CS3D_ERRBIT_NAN);
            float FX = 0.f, FY = 0.f, FZ = 0.f;
            // springs, src/propagate.cu:298-314
            const float stiff = d.E[a];
            const float4 r0 = __ldg(&d.topo.r0[i]);
            const int nbr[3] = {n0, n1, n2};
            const float r0v[3] = {r0.x, r0.y, r0.z};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float3 dd = sub3(f3(sm.xs[nbr[k]]), x);
                float R = sqrtf(dd.x * dd.x + dd.y * dd.y + dd.z * dd.z);
                float c = stiff * (R - r0v[k]) / r0v[k] / R;
                FX += c * dd.x; FY += c * dd.y; FZ += c * dd.z;
            }
            // internal pressure, src/propagate.cu:318-330 (CM of the previous step)
            {
                float4 cm = d.CM[a];
                float3 r = make_float3(x.x - cm.x, x.y - cm.y, x.z - cm.z);
                float inv = 1.0f / sqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
                float pr = 3.0f * d.press[a];
                FX += pr * (inv * r.x); FY += pr * (inv * r.y); FZ += pr * (inv * r.z);
            }
            // bond angles, src/propagate.cu:81-181 (vertex terms then arm terms)
            if (P.angles) {
                float ax = 0.f, ay = 0.f, az = 0.f;
                int o = i * 6;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    ax -= sm.armx[o + 2 * q] + sm.armx[o + 2 * q + 1];
                    ay -= sm.army[o + 2 * q] + sm.army[o + 2 * q + 1];
                    az -= sm.armz[o + 2 * q] + sm.armz[o + 2 * q + 1];
                }
                uint4 am = __ldg(&d.topo.arm[i]);
                unsigned idx[6] = {am.x & 0xffffu, am.x >> 16, am.y & 0xffffu, am.y >> 16, am.z & 0xffffu, am.z >> 16};
#pragma unroll
                for (int q = 0; q < 6; ++q) { ax += sm.armx[idx[q]]; ay += sm.army[idx[q]]; az += sm.armz[idx[q]]; }
                FX += ax; FY += ay; FZ += az;
            }
            // surface normal for the tangential friction, src/propagate.cu:558-572
            float3 A = sub3(f3(sm.xs[n1]), f3(sm.xs[n0]));
            float3 B = sub3(f3(sm.xs[n2]), f3(sm.xs[n0]));
            float3 nrm = make_float3(A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x);
            float nin = 1.0f / sqrtf(nrm.x * nrm.x + nrm.y * nrm.y + nrm.z * nrm.z);
            nrm = make_float3(sgn * (nin * nrm.x), sgn * (nin * nrm.y), sgn * (nin * nrm.z));
            // contacts
            float3 cf = make_float3(0.f, 0.f, 0.f), vt = make_float3(0.f, 0.f, 0.f);
            contact_sweep<0>(d, P, sm.sd, a, i, x, v, nrm, d.V, cf, vt);
            FX += cf.x; FY += cf.y; FZ += cf.z;
            // rigid box walls, src/propagate.cu:474-510
            if (P.rigid) {
                float g1 = x.x, g2 = __fsub_rn(P.box[0], x.x);
                if (g1 < P.thresh) FX += -P.wallk * (g1 - P.thresh);
                if (g2 < P.thresh) FX += P.wallk * (g2 - P.thresh);
                g1 = x.y; g2 = __fsub_rn(P.box[1], x.y);
                if (g1 < P.thresh) FY += -P.wallk * (g1 - P.thresh);
                if (g2 < P.thresh) FY += P.wallk * (g2 - P.thresh);
                g1 = x.z; g2 = __fsub_rn(P.box[2], x.z);
                if (g1 < P.thresh) FZ += -P.wallk * (g1 - P.thresh);
                if (g2 < P.thresh) FZ += P.wallk * (g2 - P.thresh);
            }
            // dissipative force with v after Integrate
            float3 dv = make_float3(0.f, 0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float4 vn = sm.vs[nbr[k]];
                dv.x += v.x - vn.x; dv.y += v.y - vn.y; dv.z += v.z - vn.z;
            }
            float3 fd = make_float3(-P.gint * dv.x - P.gext * vt.x - P.go * v.x,
                                    -P.gint * dv.y - P.gext * vt.y - P.go * v.y,
                                    -P.gint * dv.z - P.gext * vt.z - P.go * v.z);
            d.FC[g] = make_float4(FX, FY, FZ, 0.f);
            if (INIT) {
                d.FD[g] = make_float4(fd.x, fd.y, fd.z, 0.f);
            } else {
                const double m = P.mass;
                const float dt = P.dt;
                float vx = kick(v.x, __fmul_rn(dt, FX), m);
                float vy = kick(v.y, __fmul_rn(dt, FY), m);
                float vz = kick(v.z, __fmul_rn(dt, FZ), m);
                const double hdt = 0.5 * (double)dt;
                vx = (float)((double)vx + hdt * (double)fd.x / m);
                vy = (float)((double)vy + hdt * (double)fd.y / m);
                vz = (float)((double)vz + hdt * (double)fd.z / m);
                d.Vb[g] = make_float4(vx, vy, vz, 0.f);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// S2: second dissipative force with the updated velocities
// (src/GPUbounce.cu:1151), centre of mass (:1164), volumes and division
// flags (:1172), bounding boxes and grid extents for the next step (:1312-1334).
// ---------------------------------------------------------------------------
struct S2Smem {
    float4 xs[SLOTS];
    float4 vs[SLOTS];
    SlotData sd;
    GeomScratch gs;
};

__global__ void __launch_bounds__(SLOTS) k_s2(Dev d, int par)
{
    __shared__ S2Smem sm;
    const int W = *d.work_n;
    const int i = threadIdx.x;
    const int pn = par ^ 1;
    const uint32_t nnp = (i < NODES) ? __ldg(&d.topo.nnpack[i]) : 0u;
    const int n0 = nnp & 255, n1 = (nnp >> 8) & 255, n2 = (nnp >> 16) & 255;
    const float sgn = (float)(int8_t)(nnp >> 24);
    // per-CTA running grid extents (flushed when the instance changes)
    int acc_inst = -1;
    float acc[6];
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = d.work[w];
        const int inst = d.cell_inst[a];
        const InstParams &P = d.prm[inst];
        InstState *st = &d.st[inst];
        const size_t g = (size_t)a * SLOTS + i;
        float4 x4 = make_float4(0, 0, 0, 0), v4 = make_float4(0, 0, 0, 0);
        if (i < NODES) { x4 = d.X[g]; v4 = d.Vb[g]; }
        sm.xs[i] = x4;
        sm.vs[i] = v4;
        load_slots(d, a, P, st, par, sm.sd);
        __syncthreads();
        const float3 x = f3(x4), v = f3(v4);
        if (i < NODES) {
            float3 A = sub3(f3(sm.xs[n1]), f3(sm.xs[n0]));
            float3 B = sub3(f3(sm.xs[n2]), f3(sm.xs[n0]));
            float3 nrm = make_float3(A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x);
            float nin = 1.0f / sqrtf(nrm.x * nrm.x + nrm.y * nrm.y + nrm.z * nrm.z);
            nrm = make_float3(sgn * (nin * nrm.x), sgn * (nin * nrm.y), sgn * (nin * nrm.z));
            float3 cf = make_float3(0.f, 0.f, 0.f), vt = make_float3(0.f, 0.f, 0.f);
            contact_sweep<1>(d, P, sm.sd, a, i, x, v, nrm, d.Vb, cf, vt);
            float3 dv = make_float3(0.f, 0.f, 0.f);
            const int nbr[3] = {n0, n1, n2};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float4 vn = sm.vs[nbr[k]];
                dv.x += v.x - vn.x; dv.y += v.y - vn.y; dv.z += v.z - vn.z;
            }
            float3 fd = make_float3(-P.gint * dv.x - P.gext * vt.x - P.go * v.x,
                                    -P.gint * dv.y - P.gext * vt.y - P.go * v.y,
                                    -P.gint * dv.z - P.gext * vt.z - P.go * v.z);
            d.FD[g] = make_float4(fd.x, fd.y, fd.z, 0.f);
            d.V[g] = v4;
        }
        // centre of mass and bounding box of the post-step positions
        float3 cm;
        float4 lo, hi;
        cell_geom(sm.xs, sm.gs, cm, lo, hi);
        const bool divide_on = st->step <= P.div_steps && P.growth > 0.0f;
        if (divide_on) {
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
            }
        }
        if (i == 0) {
            d.CM[a] = make_float4(cm.x, cm.y, cm.z, 0.f);
            d.aabb[pn][2 * a] = lo;
            d.aabb[pn][2 * a + 1] = hi;
            if (inst != acc_inst) {
                if (acc_inst >= 0) {
                    int *mm = d.st[acc_inst].mm[pn];
                    for (int q = 0; q < 3; ++q) {
                        atomicMin(&mm[2 * q], f2o(acc[2 * q]));
                        atomicMax(&mm[2 * q + 1], f2o(acc[2 * q + 1]));
                    }
                }
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
    if (threadIdx.x == 0 && acc_inst >= 0) {
        int *mm = d.st[acc_inst].mm[pn];
        for (int q = 0; q < 3; ++q) {
            atomicMin(&mm[2 * q], f2o(acc[2 * q]));
            atomicMax(&mm[2 * q + 1], f2o(acc[2 * q + 1]));
        }
    }
}

// Centre of mass, bounding boxes and grid extents only (initialisation,
// src/GPUbounce.cu:739-763).
__global__ void __launch_bounds__(SLOTS) k_geom(Dev d, int par)
{
    __shared__ float4 xs[SLOTS];
    __shared__ GeomScratch gs;
    const int W = *d.work_n;
    const int i = threadIdx.x;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = d.work[w];
        const int inst = d.cell_inst[a];
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
    // count dividers
    int mine = 0;
    for (int c = threadIdx.x; c < n0; c += blockDim.x) mine += d.divflag[P.base + c] ? 1 : 0;
    mine = warp_sum(mine);
    if ((threadIdx.x & 31) == 0) atomicAdd(&cnt, mine);
    __syncthreads();
    int total = cnt;
    if (total == 0) return;
    int room = P.cap - n0;
    int ndiv = total < room ? total : room;
    if (threadIdx.x == 0) {
        if (total > room) atomicOr(&st->err, CS3D_ERRBIT_CAPACITY);
        base_slot = atomicAdd(d.div_total, ndiv);
        st->div_count = ndiv;
        st->force_rebuild = 1;
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
    // normals in ascending order (serial RNG stream)
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
        }
        st->n = n0 + ndiv;
        // grid extents of this step are recomputed after the daughters exist
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
            for (int s = 0; s < 2; ++s) {
                double sg = s == 0 ? 1.0 : -1.0;
                double n[3] = {sg * e.n[0], sg * e.n[1], sg * e.n[2]};
                double o[3] = {cm[0] + half * n[0], cm[1] + half * n[1], cm[2] + half * n[2]};
                double y[3] = {px[0] - o[0], px[1] - o[1], px[2] - o[2]};
                double dn = y[0] * n[0] + y[1] * n[1] + y[2] * n[2];
                if (dn <= 0.0) { y[0] -= dn * n[0]; y[1] -= dn * n[1]; y[2] -= dn * n[2]; }
                float4 r = make_float4((float)(y[0] + o[0]), (float)(y[1] + o[1]), (float)(y[2] + o[2]), 0.f);
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
            int wslot = atomicAdd(d.work_n, 1);
            d.work[wslot] = b;
        }
        if (i < NODES) {
            size_t ga = (size_t)a * SLOTS + i, gb = (size_t)b * SLOTS + i;
            d.X[ga] = xa;
            d.X[gb] = xb;
            d.V[gb] = d.V[ga];
            d.FC[gb] = make_float4(0, 0, 0, 0);
            d.FD[gb] = make_float4(0, 0, 0, 0);
        }
        __syncthreads();
    }
}

// G: grid extents of instances that divided this step, from all boxes.
__global__ void k_grid_fix(Dev d, int par)
{
    const int pn = par ^ 1;
    const int W = *d.work_n;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        int a = d.work[w];
        int inst = d.cell_inst[a];
        if (d.st[inst].div_count == 0) continue;
        float4 lo = d.aabb[pn][2 * a], hi = d.aabb[pn][2 * a + 1];
        int *mm = d.st[inst].mm[pn];
        atomicMin(&mm[0], f2o(lo.x)); atomicMax(&mm[1], f2o(hi.x));
        atomicMin(&mm[2], f2o(lo.y)); atomicMax(&mm[3], f2o(hi.y));
        atomicMin(&mm[4], f2o(lo.z)); atomicMax(&mm[5], f2o(hi.z));
    }
}

// ---------------------------------------------------------------------------
// Neighbour-list build (only when an instance's displacement bound reaches
// the skin, or after a division).  R1: current boxes and build extents.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SLOTS) k_nl_boxes(Dev d)
{
    if (!d.flags[0]) return;
    __shared__ float4 xs[SLOTS];
    __shared__ GeomScratch gs;
    const int W = *d.work_n;
    const int i = threadIdx.x;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = d.work[w];
        const int inst = d.cell_inst[a];
        if (!d.st[inst].rebuild) continue;  // uniform across the block
        xs[i] = (i < NODES) ? d.X[(size_t)a * SLOTS + i] : make_float4(0, 0, 0, 0);
        __syncthreads();
        float3 cm;
        float4 lo, hi;
        cell_geom(xs, gs, cm, lo, hi);
        if (i == 0) {
            d.aabb_cur[2 * a] = lo;
            d.aabb_cur[2 * a + 1] = hi;
            InstState *st = &d.st[inst];
            atomicMin(&st->bmm[0], f2o(lo.x)); atomicMax(&st->bmm[1], f2o(hi.x));
            atomicMin(&st->bmm[2], f2o(lo.y)); atomicMax(&st->bmm[3], f2o(hi.y));
            atomicMin(&st->bmm[4], f2o(lo.z)); atomicMax(&st->bmm[5], f2o(hi.z));
            float ext = fmaxf(hi.x - lo.x, fmaxf(hi.y - lo.y, hi.z - lo.z));
            atomicMax(&st->maxext, __float_as_uint(ext));
        }
        __syncthreads();
    }
}

// R2: build-grid geometry per instance and global bin offsets (one block).
__global__ void k_nl_grid(Dev d)
{
    if (!d.flags[0]) return;
    if (threadIdx.x != 0) return;
    int off = 0;
    for (int k = 0; k < d.n_inst; ++k) {
        InstState *st = &d.st[k];
        if (!st->rebuild || st->n == 0) { st->boff = off; st->bdim[0] = st->bdim[1] = st->bdim[2] = 0; continue; }
        const InstParams &P = d.prm[k];
        float h = __uint_as_float(st->maxext) + P.rlist + 1e-3f;
        int nb = 1;
        for (int q = 0; q < 3; ++q) {
            float mn = o2f(st->bmm[2 * q]), mx = o2f(st->bmm[2 * q + 1]);
            float ext = mx - mn;
            if (ext / h > 1000.0f) h = ext / 1000.0f;
        }
        for (int q = 0; q < 3; ++q) {
            float mn = o2f(st->bmm[2 * q]), mx = o2f(st->bmm[2 * q + 1]);
            int dim = (int)((mx - mn) / h) + 1;
            st->bdim[q] = dim;
            st->borg[q] = mn;
            nb *= dim;
        }
        st->bh = h;
        st->boff = off;
        off += nb;
    }
    if (off > d.bin_cap) {
        for (int k = 0; k < d.n_inst; ++k)
            if (d.st[k].rebuild) atomicOr(&d.st[k].err, CS3D_ERRBIT_GRID_OVERFLOW);
        off = 0;
        for (int k = 0; k < d.n_inst; ++k) d.st[k].rebuild = 0;
    }
    *d.total_bins = off;
}

__global__ void k_nl_zero(Dev d)
{
    if (!d.flags[0]) return;
    int tb = *d.total_bins;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= tb; b += gridDim.x * blockDim.x) d.bin_count[b] = 0;
}

__device__ __forceinline__ int build_bin(const InstState *st, float4 lo, float4 hi, int b[3])
{
    float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
    for (int q = 0; q < 3; ++q) {
        int v = (int)((c[q] - st->borg[q]) / st->bh);
        if (v < 0) v = 0;
        if (v >= st->bdim[q]) v = st->bdim[q] - 1;
        b[q] = v;
    }
    return st->boff + (b[2] * st->bdim[1] + b[1]) * st->bdim[0] + b[0];
}

__global__ void k_nl_count(Dev d)
{
    if (!d.flags[0]) return;
    const int W = *d.work_n;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        int a = d.work[w];
        const InstState *st = &d.st[d.cell_inst[a]];
        if (!st->rebuild) continue;
        int b3[3];
        int bin = build_bin(st, d.aabb_cur[2 * a], d.aabb_cur[2 * a + 1], b3);
        d.cell_bin[a] = bin;
        d.cell_rank[a] = atomicAdd(&d.bin_count[bin], 1);
    }
}

// Exclusive scan of bin counts (single block of 1024 threads).
__global__ void __launch_bounds__(1024) k_nl_scan(Dev d)
{
    if (!d.flags[0]) return;
    __shared__ int wsum[32];
    __shared__ int carry;
    const int tb = *d.total_bins;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < tb; b0 += 1024) {
        int b = b0 + threadIdx.x;
        int v = b < tb ? d.bin_count[b] : 0;
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int s = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        int excl = carry + (wid > 0 ? wsum[wid - 1] : 0) + x - v;
        if (b < tb) d.bin_start[b] = excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) d.bin_start[tb] = carry;
}

__global__ void k_nl_fill(Dev d)
{
    if (!d.flags[0]) return;
    const int W = *d.work_n;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
        int a = d.work[w];
        if (!d.st[d.cell_inst[a]].rebuild) continue;
        d.bin_cells[d.bin_start[d.cell_bin[a]] + d.cell_rank[a]] = a;
    }
}

// R7: contact-candidate cells of each cell (boxes within rlist) and the
// per-node candidate lists (nodes within rlist), deterministic order.
__global__ void __launch_bounds__(SLOTS) k_nl_build(Dev d)
{
    if (!d.flags[0]) return;
    __shared__ float4 xs[SLOTS];
    __shared__ float4 cs[SLOTS];
    __shared__ int cand[MAXC];
    __shared__ float4 clo[MAXC], chi[MAXC];
    __shared__ int ncand;
    const int W = *d.work_n;
    const int i = threadIdx.x;
    for (int w = blockIdx.x; w < W; w += gridDim.x) {
        const int a = d.work[w];
        const int inst = d.cell_inst[a];
        InstState *st = &d.st[inst];
        if (!st->rebuild) continue;
        const InstParams &P = d.prm[inst];
        const float rl = P.rlist + 1e-4f;
        const float rl2 = rl * rl;
        if (i == 0) ncand = 0;
        xs[i] = (i < NODES) ? d.X[(size_t)a * SLOTS + i] : make_float4(0, 0, 0, 0);
        __syncthreads();
        const float4 alo = d.aabb_cur[2 * a], ahi = d.aabb_cur[2 * a + 1];
        if (i < 27) {
            int b3[3];
            build_bin(st, alo, ahi, b3);
            int bx = b3[0] + (i % 3) - 1, by = b3[1] + (i / 3) % 3 - 1, bz = b3[2] + i / 9 - 1;
            if (bx >= 0 && by >= 0 && bz >= 0 && bx < st->bdim[0] && by < st->bdim[1] && bz < st->bdim[2]) {
                int bin = st->boff + (bz * st->bdim[1] + by) * st->bdim[0] + bx;
                for (int q = d.bin_start[bin]; q < d.bin_start[bin + 1]; ++q) {
                    int c = d.bin_cells[q];
                    if (c == a) continue;
                    float4 lo = d.aabb_cur[2 * c], hi = d.aabb_cur[2 * c + 1];
                    float gx = fmaxf(0.f, fmaxf(lo.x - ahi.x, alo.x - hi.x));
                    float gy = fmaxf(0.f, fmaxf(lo.y - ahi.y, alo.y - hi.y));
                    float gz = fmaxf(0.f, fmaxf(lo.z - ahi.z, alo.z - hi.z));
                    if (gx * gx + gy * gy + gz * gz >= rl2) continue;
                    int s = atomicAdd(&ncand, 1);
                    if (s < MAXC) cand[s] = c;
                }
            }
        }
        __syncthreads();
        int nc = ncand;
        if (nc > MAXC) {
            if (i == 0) atomicOr(&st->err, CS3D_ERRBIT_CAND_OVERFLOW);
            nc = MAXC;
        }
        if (i == 0) {
            // ascending cell order (insertion sort, nc <= 32)
            for (int p = 1; p < nc; ++p) {
                int v = cand[p], q = p - 1;
                while (q >= 0 && cand[q] > v) { cand[q + 1] = cand[q]; --q; }
                cand[q + 1] = v;
            }
            d.ncand[a] = nc;
            atomicMax(&st->max_cand, ncand);
        }
        __syncthreads();
        if (i < nc) {
            d.cand[a * MAXC + i] = cand[i];
            clo[i] = d.aabb_cur[2 * cand[i]];
            chi[i] = d.aabb_cur[2 * cand[i] + 1];
        }
        __syncthreads();
        const float3 x = f3(xs[i]);
        int cnt = 0;
        for (int s = 0; s < nc; ++s) {
            const int c = cand[s];
            cs[i] = (i < NODES) ? d.X[(size_t)c * SLOTS + i] : make_float4(0, 0, 0, 0);
            __syncthreads();
            if (i < NODES) {
                float4 lo = clo[s], hi = chi[s];
                float gx = fmaxf(0.f, fmaxf(lo.x - x.x, x.x - hi.x));
                float gy = fmaxf(0.f, fmaxf(lo.y - x.y, x.y - hi.y));
                float gz = fmaxf(0.f, fmaxf(lo.z - x.z, x.z - hi.z));
                if (gx * gx + gy * gy + gz * gz < rl2) {
                    for (int j = 0; j < NODES; ++j) {
                        float4 y = cs[j];
                        float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
                        if (dx * dx + dy * dy + dz * dz < rl2) {
                            if (cnt < MAXE)
                                d.ent[((size_t)a * MAXE + cnt) * SLOTS + i] = (uint16_t)((s << 8) | j);
                            ++cnt;
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (i < NODES) {
            if (cnt > MAXE) { atomicOr(&st->err, CS3D_ERRBIT_ENTRY_OVERFLOW); }
            d.nent[(size_t)a * SLOTS + i] = (uint8_t)(cnt < MAXE ? cnt : MAXE);
        }
        int wm = cnt;
        for (int o = 16; o > 0; o >>= 1) wm = max(wm, __shfl_xor_sync(0xffffffffu, wm, o));
        if ((i & 31) == 0) atomicMax(&st->max_entries, wm);
        __syncthreads();
    }
}

}  // namespace cs3d
