// cs3d_api.cu -- device context of libcs3d.so: allocation, state upload,
// the initial force evaluation, the per-step launch sequence (captured once
// per step variant into a CUDA graph) and read-back.  All entry points are
// extern "C" and return CS3D_* status codes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "cs3d_kernels.cuh"

using namespace cs3d;

struct cs3d_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int n_inst = 0;
    int cap_total = 0;
    int nsm = 148;
    std::vector<InstParams> hprm;
    std::vector<int> hn;           // host copy of the loaded cell counts
    Dev d{};
    // device allocations to free
    std::vector<void *> allocs;
    bool need_init = true;
    // The last step of the previous cs3d_step call ran S2 in fused mode: d.X and
    // d.V already hold the next step's half kick and drift, and the step-end
    // state is in d.Xe (positions) and d.Vb (velocities).
    bool prekicked = false;
    long long host_step = 0;
    int max_div_steps = 0;
    bool any_growth = false;
    bool any_com = false;          // some instance corrects its centre-of-mass motion
    bool any_far = false;          // some instance counts internal cells only (mitotic index)
    std::vector<long long> soften_steps;  // steps whose end softens cells (stiffness schedule)
    float skin = 0.1f;
    int grid_cells = 0;            // blocks of the per-cell kernels
    int grid_flat = 0;             // blocks of the per-thread kernels
    int grid_nodes = 0;            // blocks of the neighbour-list kernels
    int grid_tiles = 0;            // blocks of the bucket scan
    int grid_s2 = 0;               // blocks of S2 and the integrator
    cudaGraphExec_t graph[2][2][2][3] = {};  // [parity][division][integrate first][S2 mode: 0, fused 1, fused last 2]
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // asynchronous read-back (cs3d_get_state_async): a copy stream, two
    // device staging slots and their events
    cudaStream_t copy_stream = nullptr;
    float *astage[2] = {nullptr, nullptr};
    cudaEvent_t aready[2] = {nullptr, nullptr}, adone[2] = {nullptr, nullptr};
    bool apending[2] = {false, false};
    float last_ms = 0.f;
    long long launches_per_step = 0;
    unsigned last_err_bits = 0;
};

namespace {

#define CK(call)                                         \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) {                         \
            fprintf(stderr, "cs3d: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return CS3D_E_CUDA;                          \
        }                                                \
    } while (0)

template <typename T>
int dalloc(cs3d_ctx *c, T **p, size_t count)
{
    void *q = nullptr;
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(&q, bytes) != cudaSuccess) return CS3D_E_NOMEM;
    if (cudaMemsetAsync(q, 0, bytes, c->stream) != cudaSuccess) { cudaFree(q); return CS3D_E_CUDA; }
    c->allocs.push_back(q);
    *p = (T *)q;
    return CS3D_OK;
}

void free_all(cs3d_ctx *c)
{
    for (auto &a : c->graph)
        for (auto &b : a)
            for (auto &e : b)
                for (cudaGraphExec_t g : e)
                    if (g) cudaGraphExecDestroy(g);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    for (int q = 0; q < 2; ++q) {
        if (c->aready[q]) cudaEventDestroy(c->aready[q]);
        if (c->adone[q]) cudaEventDestroy(c->adone[q]);
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    for (void *q : c->allocs) cudaFree(q);
    c->allocs.clear();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
}

// Host copies of the mesh tables: packed neighbours, R0 and 1/R0, theta0
// with its FP64 cosine and sine, and the arm table: for node i and each of
// its neighbours n, the index n*3 + k of the arm force that the angles at
// vertex n send to i (k = the slot of i in n's neighbour list; the two
// angles at n that have i as an arm end, the NeighNeighs cases of
// src/propagate.cu:63-78).
struct TopoTables {
    uint32_t nnp[SLOTS];
    float4 r0[SLOTS], th[SLOTS];
    uint4 arm[SLOTS];
    uint8_t faces[CS3D_FACES * 7];
    double2 cs0[3 * SLOTS];
    double r0i[3 * SLOTS];
};

int topo_tables(const cs3d_topology *t, TopoTables &o)
{
    memset(&o, 0, sizeof o);
    for (int i = 0; i < 3 * SLOTS; ++i) o.cs0[i] = make_double2(1.0, 0.0);
    for (int i = 0; i < NODES; ++i) {
        int a = t->nn[i], b = t->nn[192 + i], cc = t->nn[384 + i];
        if (a < 0 || a >= NODES || b < 0 || b >= NODES || cc < 0 || cc >= NODES) return CS3D_E_ARG;
        o.nnp[i] = (uint32_t)a | ((uint32_t)b << 8) | ((uint32_t)cc << 16) | ((uint32_t)(uint8_t)(int8_t)t->sign[i] << 24);
        o.r0[i] = make_float4(t->r0[i], t->r0[192 + i], t->r0[384 + i], 0.f);
        o.th[i] = make_float4(t->theta0[3 * i], t->theta0[3 * i + 1], t->theta0[3 * i + 2], 0.f);
        for (int k = 0; k < 3; ++k) {
            const double th = (double)t->theta0[3 * i + k];
            o.cs0[3 * i + k] = make_double2(cos(th), sin(th));
            const float r0 = t->r0[k * 192 + i];
            if (!(r0 > 0.0f)) return CS3D_E_ARG;
            o.r0i[3 * i + k] = 1.0 / (double)r0;
        }
    }
    for (int i = 0; i < NODES; ++i) {
        unsigned idx[3];
        for (int q = 0; q < 3; ++q) {
            const int n = t->nn[q * 192 + i];
            int k = -1;
            for (int m = 0; m < 3; ++m)
                if (t->nn[m * 192 + n] == i) k = m;
            if (k < 0) return CS3D_E_ARG;  // neighbour table not symmetric
            idx[q] = (unsigned)(n * 3 + k);
        }
        o.arm[i] = make_uint4(idx[0], idx[1], idx[2], 0u);
    }
    for (int f = 0; f < CS3D_FACES * 7; ++f) {
        if (t->faces[f] < 0 || t->faces[f] >= NODES) return CS3D_E_ARG;
        o.faces[f] = (uint8_t)t->faces[f];
    }
    return CS3D_OK;
}

int upload_topology(cs3d_ctx *c, const cs3d_topology *t)
{
    TopoTables tt;
    int rc = topo_tables(t, tt);
    if (rc) return rc;
    Topo &T = c->d.topo;
    if ((rc = dalloc(c, &T.cs0, 3 * SLOTS))) return rc;
    if ((rc = dalloc(c, &T.r0i, 3 * SLOTS))) return rc;
    if ((rc = dalloc(c, &T.nnpack, SLOTS))) return rc;
    if ((rc = dalloc(c, &T.r0, SLOTS))) return rc;
    if ((rc = dalloc(c, &T.th0, SLOTS))) return rc;
    if ((rc = dalloc(c, &T.arm, SLOTS))) return rc;
    if ((rc = dalloc(c, &T.faces, CS3D_FACES * 7))) return rc;
    CK(cudaMemcpyAsync(T.cs0, tt.cs0, sizeof tt.cs0, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.r0i, tt.r0i, sizeof tt.r0i, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.nnpack, tt.nnp, sizeof tt.nnp, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.r0, tt.r0, sizeof tt.r0, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.th0, tt.th, sizeof tt.th, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.arm, tt.arm, sizeof tt.arm, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(T.faces, tt.faces, sizeof tt.faces, cudaMemcpyHostToDevice, c->stream));
    // the host tables go out of scope: the copies must have completed
    CK(cudaStreamSynchronize(c->stream));
    return CS3D_OK;
}

InstParams make_inst(const cs3d_params &p, int base, int cap, float skin)
{
    InstParams q{};
    q.mass = p.particle_mass;
    q.mass_d = (double)p.particle_mass;
    q.inv_m = 1.0 / (double)p.particle_mass;   // IEEE division on the host: correctly rounded
    q.rr = p.repulsion_range;
    q.ra = p.attraction_range;
    q.rs = p.repulsion_strength;
    q.as = p.attraction_strength;
    q.E = p.youngs_mod;
    q.stiff1 = p.stiffness1;
    q.gint = p.internal_damping;
    q.gext = p.viscotic_damping;
    q.go = p.gamma_visc;
    q.divvol = p.division_vol;
    q.dt = p.time_interval;
    q.maxp = p.max_pressure;
    q.minp = p.min_pressure;
    q.growth = p.growth_rate;
    q.thresh = p.thresh_dist;
    for (int k = 0; k < 3; ++k) q.box[k] = p.box_len[k];
    volatile float ra = p.attraction_range;  // float products, no contraction
    q.ra2 = ra * ra;
    volatile float as = p.attraction_strength, E = p.youngs_mod, rs = p.repulsion_strength;
    q.asE = as * E;
    q.rsE = rs * E;
    q.wallk = 100.0f * E;
    q.skin = skin;
    q.skin_base = skin;
    q.rlist = p.attraction_range + skin;
    q.check_sph = p.check_sphericity;
    q.angles = p.constrain_angles;
    q.rigid = p.use_rigid_box;
    q.daught_same = p.daught_same_stiffness;
    q.div_steps = p.div_time_steps;
    q.base = base;
    q.cap = cap;
    q.rands = p.add_rands ? 1 : 0;
    q.rscale = p.rand_scale_factor;
    q.rdt = sqrtf(p.time_interval);
    q.rseed = (unsigned)p.rand_seed;
    q.correct_com = p.correct_com ? 1 : 0;
    q.diffE = p.use_different_stiffnesses ? 1 : 0;
    q.E2 = p.stiffness2;
    q.phase = p.phase_count;
    q.soften = p.use_different_stiffnesses && p.soften_after_growth ? 1 : 0;
    q.soft_n = p.number_of_softer_cells;
    q.soft_frac = p.fraction_of_softer_cells;
    q.soft_rand = p.choose_random_cell_indices ? 1 : 0;
    q.closeness = p.closeness_to_center;
    q.far_r = p.count_internal_radius > 0.0f ? p.count_internal_radius : 0.0f;
    return q;
}

int check_params(const cs3d_params &p)
{
    if (!(p.particle_mass > 0) || !(p.time_interval > 0) || !(p.attraction_range > 0) ||
        !(p.repulsion_range >= 0))
        return CS3D_E_CONFIG;
    return CS3D_OK;
}

// Staged SoA (6 arrays of k floats) -> float4 positions (and velocities);
// padding nodes (180..191 of each cell) are left zero.
__global__ void k_pack(const float *stage, float4 *X, float4 *V, size_t k)
{
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < k; g += (size_t)gridDim.x * blockDim.x) {
        if (g % SLOTS >= NODES) continue;
        X[g] = make_float4(stage[g], stage[k + g], stage[2 * k + g], 0.f);
        if (V) V[g] = make_float4(stage[3 * k + g], stage[4 * k + g], stage[5 * k + g], 0.f);
    }
}

// float4 arrays a, b -> staged SoA components (a.xyz, b.xyz).
__global__ void k_unpack(float *stage, const float4 *a, const float4 *b, size_t k)
{
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < k; g += (size_t)gridDim.x * blockDim.x) {
        if (a) { const float4 v = a[g]; stage[g] = v.x; stage[k + g] = v.y; stage[2 * k + g] = v.z; }
        if (b) { const float4 v = b[g]; stage[3 * k + g] = v.x; stage[4 * k + g] = v.y; stage[5 * k + g] = v.z; }
    }
}

// Rebuild the active-cell work table from the device cell counts.
__global__ void k_build_work(Dev d)
{
    __shared__ int off;
    if (threadIdx.x == 0) off = 0;
    __syncthreads();
    for (int k = 0; k < d.n_inst; ++k) {
        int n = d.st[k].n, base = d.prm[k].base;
        for (int c = threadIdx.x; c < n; c += blockDim.x) d.work[off + c] = base + c;
        __syncthreads();
        if (threadIdx.x == 0) off += n;
        __syncthreads();
    }
    if (threadIdx.x == 0) *d.work_n = off;
}

// Optional per-launch event recording (profiling pass of cs3d_profile_step).
struct Prof {
    std::vector<cudaEvent_t> *ev = nullptr;
    std::vector<const char *> *names = nullptr;
    void mark(cudaStream_t s, const char *name) const {
        if (!ev) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        ev->push_back(e);
        names->push_back(name);
    }
};

// Neighbour-list build: spatial hash of the nodes (counting sort by
// bucket), then the per-cell lists.  Every kernel returns at once when no
// instance rebuilds this step.
int launch_nl_kernels(const Dev &d, cudaStream_t s, int grid_nodes, int grid_tiles, const Prof &pf = Prof())
{
    k_nh_zero<<<grid_tiles, 256, 0, s>>>(d); pf.mark(s, "nh_zero");
    k_nh_count<<<grid_nodes, SLOTS, 0, s>>>(d); pf.mark(s, "nh_count");
    k_nh_scan_tiles<<<grid_tiles, 256, 0, s>>>(d); pf.mark(s, "nh_scan_tiles");
    k_nh_scan_top<<<1, 1024, 0, s>>>(d); pf.mark(s, "nh_scan_top");
    k_nh_scan_apply<<<grid_tiles, 256, 0, s>>>(d); pf.mark(s, "nh_scan_apply");
    k_nh_fill<<<grid_nodes, SLOTS, 0, s>>>(d); pf.mark(s, "nh_fill");
    k_nl_cell<<<grid_nodes, SLOTS, 0, s>>>(d, 0); pf.mark(s, "nl_cell");
    k_nl_cell<<<grid_nodes, SLOTS, 0, s>>>(d, 1); pf.mark(s, "nl_cell_nbr");
    CK(cudaGetLastError());
    return CS3D_OK;
}
constexpr int NL_LAUNCHES = 8;

int launch_nl_build(cs3d_ctx *c, const Prof &pf = Prof())
{
    return launch_nl_kernels(c->d, c->stream, c->grid_nodes, c->grid_tiles, pf);
}

// Buckets of the node hash for a capacity of `cells` cells.
constexpr int hash_size(long long cells)
{
    long long n = std::max<long long>(cells * SLOTS, SCAN_TILE);
    int h = SCAN_TILE;
    while (h < n) h <<= 1;
    return h;
}

int run_init(cs3d_ctx *c)
{
    const Dev &d = c->d;
    cudaStream_t s = c->stream;
    k_build_work<<<1, 256, 0, s>>>(d);
    k_init_begin<<<1, 256, 0, s>>>(d);
    k_geom<<<c->grid_cells, SLOTS, 0, s>>>(d, 0);
    // correct_com at set-up (src/GPUbounce.cu:785-805): after the first grid,
    // before the first force evaluation
    if (c->any_com) k_com_shift<<<c->n_inst, 256, 0, s>>>(d);
    CK(cudaGetLastError());
    int rc = launch_nl_build(c);
    if (rc) return rc;
    k_s1<true><<<c->grid_cells, SLOTS, sizeof(S1Smem), s>>>(d, 0);
    CK(cudaGetLastError());
    c->host_step = 0;
    c->need_init = false;
    return CS3D_OK;
}

// One timestep, src/GPUbounce.cu:1055-1338, as a fixed launch sequence.
// k1: the step starts with k_integrate (else the previous step's fused S2
// did it); fuse: S2 also integrates the next step (1: the next step follows in
// the same call; 2: the last step of a call, which also keeps the step-end
// positions for the read-back; on division steps the two cells of each
// division are integrated after their placement); soften: the number of this
// step when its end softens cells (launched outside the graphs), else 0.
int launch_step(cs3d_ctx *c, int par, bool div, bool k1 = true, int fuse = 0, const Prof &pf = Prof(),
                long long soften = 0)
{
    const Dev &d = c->d;
    cudaStream_t s = c->stream;
    int n = 0;
    if (k1) { k_integrate<<<c->grid_s2, SLOTS, 0, s>>>(d); ++n; pf.mark(s, "integrate"); }
    k_step_begin<<<1, 256, 0, s>>>(d, par ^ 1); ++n; pf.mark(s, "step_begin");
    int rc = launch_nl_build(c, pf);
    if (rc) return rc;
    n += NL_LAUNCHES;
    k_s1<false><<<c->grid_cells, SLOTS, sizeof(S1Smem), s>>>(d, par); ++n; pf.mark(s, "s1_con_dis");
    if (div && fuse == 2) k_s2<true, 2><<<c->grid_s2, SLOTS, 0, s>>>(d, par);
    else if (div && fuse) k_s2<true, 1><<<c->grid_s2, SLOTS, 0, s>>>(d, par);
    else if (div) k_s2<true, 0><<<c->grid_s2, SLOTS, 0, s>>>(d, par);
    else if (fuse == 2) k_s2<false, 2><<<c->grid_s2, SLOTS, 0, s>>>(d, par);
    else if (fuse) k_s2<false, 1><<<c->grid_s2, SLOTS, 0, s>>>(d, par);
    else k_s2<false, 0><<<c->grid_s2, SLOTS, 0, s>>>(d, par);
    ++n; pf.mark(s, fuse ? "s2_dis_geom_integrate" : "s2_dis_geom");
    if (div) {
        k_div_select<<<c->n_inst, 256, 0, s>>>(d, par); ++n; pf.mark(s, "div_select");
        k_div_apply<<<c->grid_cells, SLOTS, 0, s>>>(d, par); ++n; pf.mark(s, "div_apply");
        k_grid_fix<<<c->grid_flat, 256, 0, s>>>(d, par); ++n; pf.mark(s, "grid_fix");
        if (c->any_far) { k_far_count<<<c->n_inst, 32, 0, s>>>(d); ++n; pf.mark(s, "far_count"); }
        // S2 did the next half kick of every cell that does not divide
        if (fuse) { k_integrate_divided<<<c->grid_cells, SLOTS, 0, s>>>(d); ++n; pf.mark(s, "integrate_divided"); }
    }
    if (soften) { k_soften<<<c->n_inst, 32, 0, s>>>(d, (int)soften); ++n; pf.mark(s, "soften"); }
    if (c->any_com) { k_com_shift<<<c->n_inst, 256, 0, s>>>(d); ++n; pf.mark(s, "com_shift"); }
    CK(cudaGetLastError());
    c->launches_per_step = n;
    return CS3D_OK;
}

bool is_soften_step(const cs3d_ctx *c, long long s)
{
    return std::find(c->soften_steps.begin(), c->soften_steps.end(), s) != c->soften_steps.end();
}

int get_graph(cs3d_ctx *c, int par, bool div, bool k1, int fuse, cudaGraphExec_t *out)
{
    cudaGraphExec_t &g = c->graph[par][div ? 1 : 0][k1 ? 1 : 0][fuse];
    if (!g) {
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = launch_step(c, par, div, k1, fuse);
        cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
        if (rc) { if (e == cudaSuccess) cudaGraphDestroy(graph); return rc; }
        CK(e);
        e = cudaGraphInstantiate(&g, graph, 0);
        cudaGraphDestroy(graph);
        CK(e);
    }
    *out = g;
    return CS3D_OK;
}

int ensure_init(cs3d_ctx *c)
{
    if (!c->need_init) return CS3D_OK;
    return run_init(c);
}

// After a fused last step d.X and d.V hold the next step's half kick and
// drift; copy the kept step-end state (d.Xe, d.Vb) back for the operations
// that read or rebuild from d.X and d.V (the forces and pressures are those of
// the finished step either way).  The next step then runs k_integrate again.
int settle(cs3d_ctx *c)
{
    if (!c->prekicked) return CS3D_OK;
    const size_t bytes = sizeof(float4) * (size_t)c->cap_total * SLOTS;
    CK(cudaMemcpyAsync(c->d.X, c->d.Xe, bytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d.V, c->d.Vb, bytes, cudaMemcpyDeviceToDevice, c->stream));
    c->prekicked = false;
    return CS3D_OK;
}

int read_errors(cs3d_ctx *c, unsigned *any)
{
    std::vector<InstState> st(c->n_inst);
    CK(cudaMemcpyAsync(st.data(), c->d.st, sizeof(InstState) * c->n_inst, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    unsigned bits = 0;
    for (auto &q : st) bits |= q.err;
    *any = bits;
    c->last_err_bits = bits;
    return CS3D_OK;
}

int inst_count(cs3d_ctx *c, int inst, int *n)
{
    int v = 0;
    CK(cudaMemcpyAsync(&v, &c->d.st[inst].n, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *n = v;
    return CS3D_OK;
}

// Host <-> device transfers of 192-stride SoA node arrays go through a
// device staging area (c->d.stage, 6 arrays of cap*192 floats): the host
// copies move the caller's arrays as they are (at full PCIe speed when the
// caller's memory is pinned) and kernels convert to and from the float4
// layout.

// Gather up to two float4 arrays of instance inst (n cells) into staged
// SoA components (k = 0..5 -> a.x, a.y, a.z, b.x, b.y, b.z), then copy the
// requested ones to the host.
int fetch_soa(cs3d_ctx *c, int inst, int n, const float4 *a, const float4 *b, float *const out[6])
{
    if (n == 0) return CS3D_OK;
    const size_t k = (size_t)n * SLOTS;
    const size_t off = (size_t)c->hprm[inst].base * SLOTS;
    k_unpack<<<c->grid_flat, 256, 0, c->stream>>>(c->d.stage, a ? a + off : nullptr, b ? b + off : nullptr, k);
    CK(cudaGetLastError());
    for (int q = 0; q < 6; ++q)
        if (out[q]) CK(cudaMemcpyAsync(out[q], c->d.stage + (size_t)q * k, sizeof(float) * k, cudaMemcpyDeviceToHost,
                                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CS3D_OK;
}

}  // namespace

extern "C" {

int cs3d_create_ensemble(int n_inst, const cs3d_params *params, const cs3d_topology *topo,
                         const int *capacity, int device, void *stream, cs3d_ctx **out)
{
    if (!out || !params || !topo || !capacity || n_inst <= 0) return CS3D_E_ARG;
    *out = nullptr;
    long long total = 0;
    for (int k = 0; k < n_inst; ++k) {
        if (capacity[k] <= 0) return CS3D_E_ARG;
        if (check_params(params[k])) return CS3D_E_CONFIG;
        total += capacity[k];
    }
    if (total > (1 << 23)) return CS3D_E_ARG;  // cell ids are packed in 24 bits for pair records
    if (total * SLOTS * 2 > (1ll << 31) - SCAN_TILE) return CS3D_E_ARG;  // int bucket offsets of the node hash
    cs3d_ctx *c = new (std::nothrow) cs3d_ctx();
    if (!c) return CS3D_E_NOMEM;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return CS3D_E_CUDA; }
    if (stream) c->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return CS3D_E_CUDA; }
        c->own_stream = true;
    }
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
    c->n_inst = n_inst;
    c->cap_total = (int)total;
    c->hn.assign(n_inst, 0);
    int base = 0;
    for (int k = 0; k < n_inst; ++k) {
        c->hprm.push_back(make_inst(params[k], base, capacity[k], c->skin));
        base += capacity[k];
        if (params[k].growth_rate > 0) c->any_growth = true;
        if (params[k].correct_com) c->any_com = true;
        if (params[k].count_internal_radius > 0) c->any_far = true;
        if (params[k].use_different_stiffnesses && params[k].soften_after_growth) {
            const long long s = (long long)params[k].div_time_steps + 2;
            if (std::find(c->soften_steps.begin(), c->soften_steps.end(), s) == c->soften_steps.end())
                c->soften_steps.push_back(s);
        }
        c->max_div_steps = std::max(c->max_div_steps, params[k].div_time_steps);
    }
    Dev &d = c->d;
    d.n_inst = n_inst;
    d.single = n_inst == 1 ? 1 : 0;
    d.cap_total = c->cap_total;
    const size_t nodes = (size_t)c->cap_total * SLOTS;
    int rc = CS3D_OK;
#define AL(ptr, cnt) if (!rc) rc = dalloc(c, &(ptr), (cnt))
    AL(d.prm, n_inst);
    AL(d.st, n_inst);
    AL(d.X, nodes); AL(d.V, nodes); AL(d.Vb, nodes); AL(d.FC, nodes); AL(d.FD, nodes); AL(d.FR, nodes);
    AL(d.Xe, nodes);
    AL(d.stage, 6 * nodes);
    AL(d.CM, c->cap_total);
    AL(d.press, c->cap_total); AL(d.E, c->cap_total); AL(d.vol, c->cap_total); AL(d.area, c->cap_total);
    AL(d.divflag, c->cap_total);
    AL(d.aabb[0], 2 * (size_t)c->cap_total); AL(d.aabb[1], 2 * (size_t)c->cap_total);
    AL(d.cell_inst, c->cap_total);
    AL(d.work, c->cap_total); AL(d.work_n, 1);
    AL(d.cand, (size_t)c->cap_total * MAXC); AL(d.ncand, c->cap_total);
    AL(d.dlist, (size_t)c->cap_total * MAXD * SLOTS); AL(d.ndis, nodes); AL(d.dirty, c->cap_total);
    AL(d.Xb, nodes);
    AL(d.ent, (size_t)c->cap_total * MAXE * SLOTS); AL(d.nent, nodes);
    d.hsize = hash_size(2ll * c->cap_total);  // slices: a power of two >= nodes per instance
    AL(d.hcount, (size_t)d.hsize + SCAN_TILE); AL(d.hscan, (size_t)d.hsize / SCAN_TILE + 1); AL(d.hsz, 1);
    AL(d.hpos, nodes); AL(d.node_rank, nodes);
    AL(d.divtab, c->cap_total); AL(d.div_total, 1);
    d.ev_cap = std::max(1 << 16, 2 * c->cap_total);
    AL(d.events, d.ev_cap); AL(d.n_events, 1);
    d.far_cap = d.ev_cap;
    AL(d.farlog, d.far_cap); AL(d.n_far, 1);
    AL(d.pick, (size_t)c->cap_total + n_inst);
    AL(d.flags, 4);
    d.pair_cap = 1;
    AL(d.pairs, 1); AL(d.n_pairs, 1);
#undef AL
    if (!rc) rc = upload_topology(c, topo);
    if (rc) { free_all(c); delete c; return rc; }
    // instance parameters, RANMAR streams and slot ownership
    std::vector<InstState> st(n_inst);
    std::vector<int> owner(c->cap_total);
    for (int k = 0; k < n_inst; ++k) {
        memset(&st[k], 0, sizeof(InstState));
        cs3d_rng r;
        if (cs3d_rng_init(&r, params[k].rng_ij, params[k].rng_kl) != CS3D_OK) {
            free_all(c); delete c; return CS3D_E_CONFIG;
        }
        memcpy(st[k].u, r.u, sizeof r.u);
        st[k].syscm[0] = st[k].syscm[1] = st[k].syscm[2] = 1.0f;   // src/GPUbounce.cu:240
        st[k].rc = r.c; st[k].rcd = r.cd; st[k].rcm = r.cm; st[k].i97 = r.i97; st[k].j97 = r.j97;
        for (int q = 0; q < capacity[k]; ++q) owner[c->hprm[k].base + q] = k;
    }
    if (cudaMemcpyAsync(d.prm, c->hprm.data(), sizeof(InstParams) * n_inst, cudaMemcpyHostToDevice, c->stream) ||
        cudaMemcpyAsync(d.st, st.data(), sizeof(InstState) * n_inst, cudaMemcpyHostToDevice, c->stream) ||
        cudaMemcpyAsync(d.cell_inst, owner.data(), sizeof(int) * owner.size(), cudaMemcpyHostToDevice, c->stream) ||
        cudaEventCreate(&c->ev0) || cudaEventCreate(&c->ev1) || cudaStreamSynchronize(c->stream)) {
        free_all(c); delete c; return CS3D_E_CUDA;
    }
    int occ = 1;
    if (cudaFuncSetAttribute(k_s1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(S1Smem)) ||
        cudaFuncSetAttribute(k_s1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(S1Smem))) {
        free_all(c); delete c; return CS3D_E_CUDA;
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_s1<false>, SLOTS, sizeof(S1Smem));
    c->grid_cells = std::max(1, std::min(c->cap_total, c->nsm * std::max(occ, 1)));
    c->grid_flat = std::max(1, std::min((c->cap_total + 255) / 256 + 1, c->nsm * 8));
    int occ_nl = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_nl, k_nl_cell, SLOTS, 0);
    c->grid_nodes = std::max(1, std::min(c->cap_total, c->nsm * std::max(occ_nl, 1)));
    c->grid_tiles = std::max(1, std::min(d.hsize / SCAN_TILE + 1, c->nsm * 8));
    int occ_s2 = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s2, k_s2<true, 0>, SLOTS, 0);
    c->grid_s2 = std::max(1, std::min(c->cap_total, c->nsm * std::max(occ_s2, 1)));
    *out = c;
    return CS3D_OK;
}

int cs3d_create(const cs3d_params *params, const cs3d_topology *topo, int capacity_cells, int device,
                void *stream, cs3d_ctx **out)
{
    return cs3d_create_ensemble(1, params, topo, &capacity_cells, device, stream, out);
}

int cs3d_destroy(cs3d_ctx *c)
{
    if (!c) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
    return CS3D_OK;
}

int cs3d_set_skin_schedule(cs3d_ctx *c, int n, const int *min_cells, const float *skins)
{
    if (!c || n < 0 || n > CS3D_SKIN_RANGES || (n > 0 && (!min_cells || !skins))) return CS3D_E_ARG;
    for (int k = 0; k < n; ++k) {
        if (min_cells[k] < 1 || (k > 0 && min_cells[k] <= min_cells[k - 1])) return CS3D_E_ARG;
        if (!(skins[k] > 0.002f) || skins[k] > 1.0f) return CS3D_E_ARG;
    }
    cudaSetDevice(c->device);
    for (auto &q : c->hprm) {
        q.sk_n = n;
        for (int k = 0; k < CS3D_SKIN_RANGES; ++k) {
            q.sk_min[k] = k < n ? min_cells[k] : 0;
            q.sk_val[k] = k < n ? skins[k] : 0.0f;
        }
    }
    // only the schedule fields: the device keeps the skin in use (and so
    // its lists) until the next step compares it with the schedule
    for (int k = 0; k < c->n_inst; ++k) {
        InstParams *dp = c->d.prm + k;
        const InstParams &hp = c->hprm[k];
        CK(cudaMemcpyAsync(&dp->sk_n, &hp.sk_n, sizeof hp.sk_n, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(dp->sk_min, hp.sk_min, sizeof hp.sk_min, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(dp->sk_val, hp.sk_val, sizeof hp.sk_val, cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return CS3D_OK;
}

int cs3d_set_option(cs3d_ctx *c, int option, long long value)
{
    if (!c) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    switch (option) {
    case CS3D_OPT_RECORD_PAIRS:
        c->d.record_pairs = value ? 1 : 0;
        break;
    case CS3D_OPT_HALO_STATS:
        c->d.halo_stats = value ? 1 : 0;
        break;
    case CS3D_OPT_PAIR_CAPACITY: {
        if (value < 1) return CS3D_E_ARG;
        int4 *p = nullptr;
        if (cudaMalloc(&p, sizeof(int4) * (size_t)value) != cudaSuccess) return CS3D_E_NOMEM;
        c->allocs.push_back(p);
        int4 *old = c->d.pairs;
        c->d.pairs = p;
        c->d.pair_cap = value;
        // the previous buffer is released once the work queued on it is done
        CK(cudaStreamSynchronize(c->stream));
        const auto it = std::find(c->allocs.begin(), c->allocs.end(), (void *)old);
        if (it != c->allocs.end()) {
            c->allocs.erase(it);
            cudaFree(old);
        }
        break;
    }
    case CS3D_OPT_SKIN: {
        float s = (float)value * 1e-6f;
        if (!(s > 0.002f) || s > 1.0f) return CS3D_E_ARG;
        if (int rc = settle(c)) return rc;   // the re-initialisation starts from the step-end state
        c->skin = s;
        for (auto &q : c->hprm) { q.skin = s; q.skin_base = s; q.rlist = q.ra + s; }
        CK(cudaMemcpyAsync(c->d.prm, c->hprm.data(), sizeof(InstParams) * c->n_inst, cudaMemcpyHostToDevice, c->stream));
        c->need_init = true;
        break;
    }
    case CS3D_OPT_REBUILD: {
        if (int rc = ensure_init(c)) return rc;
        k_force_rebuild<<<1, 256, 0, c->stream>>>(c->d);
        CK(cudaGetLastError());
        return CS3D_OK;  // no launch parameter changed: the graphs stay valid
    }
    default:
        return CS3D_E_ARG;
    }
    // launch parameters are baked into captured graphs: drop them
    for (auto &a : c->graph)
        for (auto &b : a)
            for (auto &e : b)
                for (cudaGraphExec_t &g : e)
                    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    return CS3D_OK;
}

int cs3d_load_state(cs3d_ctx *c, int inst, int n, const float *X, const float *Y, const float *Z,
                    const float *VX, const float *VY, const float *VZ, const float *pressure,
                    const float *youngs)
{
    if (!c || inst < 0 || inst >= c->n_inst || n < 0 || (n > 0 && (!X || !Y || !Z))) return CS3D_E_ARG;
    const InstParams &P = c->hprm[inst];
    if (n > P.cap) return CS3D_E_CAPACITY;
    cudaSetDevice(c->device);
    // the other instances back to their step-end state: the re-initialisation
    // that follows a load starts from it
    if (int rc = settle(c)) return rc;
    const size_t slots = (size_t)P.cap * SLOTS;
    const size_t k = (size_t)n * SLOTS;
    const size_t off0 = (size_t)P.base * SLOTS;
    const Dev &d0 = c->d;
    // the caller's SoA arrays into the staging area, packed on the device
    const float *in[6] = {X, Y, Z, VX, VY, VZ};
    const bool with_v = VX && VY && VZ;
    for (int q = 0; q < (with_v ? 6 : 3); ++q)
        if (k) CK(cudaMemcpyAsync(d0.stage + (size_t)q * k, in[q], sizeof(float) * k, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(d0.X + off0, 0, sizeof(float4) * slots, c->stream));
    CK(cudaMemsetAsync(d0.V + off0, 0, sizeof(float4) * slots, c->stream));
    if (k) k_pack<<<c->grid_flat, 256, 0, c->stream>>>(d0.stage, d0.X + off0, with_v ? d0.V + off0 : nullptr, k);
    CK(cudaGetLastError());
    std::vector<float> p(P.cap, 0.f), e(P.cap, 0.f);
    for (int k = 0; k < n; ++k) {
        p[k] = pressure ? pressure[k] : P.minp;
        e[k] = youngs ? youngs[k] : P.stiff1;
    }
    const size_t off = off0;
    const Dev &d = c->d;
    CK(cudaMemsetAsync(d.Vb + off, 0, sizeof(float4) * slots, c->stream));
    CK(cudaMemsetAsync(d.FC + off, 0, sizeof(float4) * slots, c->stream));
    CK(cudaMemsetAsync(d.FD + off, 0, sizeof(float4) * slots, c->stream));
    CK(cudaMemsetAsync(d.CM + P.base, 0, sizeof(float4) * P.cap, c->stream));
    CK(cudaMemsetAsync(d.vol + P.base, 0, sizeof(float) * P.cap, c->stream));
    CK(cudaMemsetAsync(d.area + P.base, 0, sizeof(float) * P.cap, c->stream));
    CK(cudaMemsetAsync(d.divflag + P.base, 0, P.cap, c->stream));
    CK(cudaMemcpyAsync(d.press + P.base, p.data(), sizeof(float) * P.cap, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d.E + P.base, e.data(), sizeof(float) * P.cap, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(&d.st[inst].n, &n, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    int zero = 0;
    CK(cudaMemcpyAsync(&d.st[inst].step, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(&d.st[inst].err, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    static const float one3[3] = {1.0f, 1.0f, 1.0f};   // the reference's initial system centre
    CK(cudaMemcpyAsync(d.st[inst].syscm, one3, sizeof one3, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->hn[inst] = n;
    c->need_init = true;
    return CS3D_OK;
}

int cs3d_set_rng(cs3d_ctx *c, int inst, const cs3d_rng *r)
{
    if (!c || !r || inst < 0 || inst >= c->n_inst || !r->ok) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    InstState st;
    CK(cudaMemcpyAsync(&st, &c->d.st[inst], sizeof st, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    memcpy(st.u, r->u, sizeof st.u);
    st.rc = r->c; st.rcd = r->cd; st.rcm = r->cm; st.i97 = r->i97; st.j97 = r->j97;
    CK(cudaMemcpyAsync(&c->d.st[inst], &st, sizeof st, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CS3D_OK;
}

int cs3d_get_rng(cs3d_ctx *c, int inst, cs3d_rng *r)
{
    if (!c || !r || inst < 0 || inst >= c->n_inst) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    InstState st;
    CK(cudaMemcpyAsync(&st, &c->d.st[inst], sizeof st, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    memset(r, 0, sizeof *r);
    memcpy(r->u, st.u, sizeof r->u);
    r->c = st.rc; r->cd = st.rcd; r->cm = st.rcm; r->i97 = st.i97; r->j97 = st.j97;
    r->ok = 1;
    return CS3D_OK;
}

int cs3d_step(cs3d_ctx *c, int n_steps)
{
    if (!c || n_steps < 0) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev0, c->stream));
    // the previous call's last S2 may already have done this step's half
    // kick and drift
    bool k1 = !c->prekicked;
    for (int k = 0; k < n_steps; ++k) {
        long long s = c->host_step + 1;
        int par = (int)((s - 1) & 1);
        bool div = c->any_growth && s <= c->max_div_steps;
        const bool soften = is_soften_step(c, s);
        // S2 integrates the next step unless the step shifts or softens
        // cells after S2 (CoM correction, growth-end softening); on the last
        // step of the call it also keeps the step-end positions
        const int fuse = (c->any_com || soften) ? 0 : (k + 1 < n_steps ? 1 : 2);
        if (soften) {
            // the one step that softens cells runs outside the graphs
            if ((rc = launch_step(c, par, div, k1, 0, Prof(), s))) return rc;
        } else {
            cudaGraphExec_t g;
            if ((rc = get_graph(c, par, div, k1, fuse, &g))) return rc;
            CK(cudaGraphLaunch(g, c->stream));
        }
        c->host_step = s;
        k1 = fuse == 0;
        c->prekicked = fuse == 2;
    }
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    CK(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
    unsigned bits = 0;
    if ((rc = read_errors(c, &bits))) return rc;
    if (bits & CS3D_ERRBIT_CAPACITY) return CS3D_E_CAPACITY;
    if (bits) return CS3D_E_DEVICE_FLAGS;
    return CS3D_OK;
}

int cs3d_profile_step(cs3d_ctx *c, int n_steps, float *kernel_ms, char *names, int names_len,
                      int max_kernels, int *n_kernels)
{
    if (!c || n_steps <= 0 || !n_kernels) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    // every profiled step launches the same kernels, k_integrate first
    if ((rc = settle(c))) return rc;
    std::vector<double> acc;
    std::vector<const char *> first_names;
    for (int k = 0; k < n_steps; ++k) {
        long long st = c->host_step + 1;
        int par = (int)((st - 1) & 1);
        bool div = c->any_growth && st <= c->max_div_steps;
        std::vector<cudaEvent_t> ev;
        std::vector<const char *> nm;
        Prof pf;
        pf.ev = &ev;
        pf.names = &nm;
        cudaEvent_t e0;
        CK(cudaEventCreate(&e0));
        CK(cudaEventRecord(e0, c->stream));
        if ((rc = launch_step(c, par, div, true, 0, pf, is_soften_step(c, st) ? st : 0))) return rc;
        c->host_step = st;
        CK(cudaEventSynchronize(ev.empty() ? e0 : ev.back()));
        if (acc.size() < ev.size()) { acc.resize(ev.size(), 0.0); first_names = nm; }
        cudaEvent_t prev = e0;
        for (size_t q = 0; q < ev.size(); ++q) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, prev, ev[q]);
            acc[q] += ms;
            prev = ev[q];
        }
        cudaEventDestroy(e0);
        for (auto e : ev) cudaEventDestroy(e);
    }
    int nk = (int)acc.size();
    *n_kernels = nk;
    std::string all;
    for (int q = 0; q < nk; ++q) {
        if (kernel_ms && q < max_kernels) kernel_ms[q] = (float)(acc[q] / n_steps);
        if (q) all += ",";
        all += first_names[q];
    }
    if (names && names_len > 0) snprintf(names, (size_t)names_len, "%s", all.c_str());
    unsigned bits = 0;
    if ((rc = read_errors(c, &bits))) return rc;
    return bits ? CS3D_E_DEVICE_FLAGS : CS3D_OK;
}

int cs3d_last_step_ms(cs3d_ctx *c, float *ms)
{
    if (!c || !ms) return CS3D_E_ARG;
    *ms = c->last_ms;
    return CS3D_OK;
}

int cs3d_get_state(cs3d_ctx *c, int inst, int *n_cells, float *X, float *Y, float *Z, float *VX, float *VY,
                   float *VZ, float *pressure, float *youngs)
{
    if (!c || inst < 0 || inst >= c->n_inst) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    int n = 0;
    if ((rc = inst_count(c, inst, &n))) return rc;
    if (n_cells) *n_cells = n;
    if (X || Y || Z || VX || VY || VZ) {
        float *const out[6] = {X, Y, Z, VX, VY, VZ};
        const float4 *xs = c->prekicked ? c->d.Xe : c->d.X, *vs = c->prekicked ? c->d.Vb : c->d.V;
        if ((rc = fetch_soa(c, inst, n, (X || Y || Z) ? xs : nullptr, (VX || VY || VZ) ? vs : nullptr, out)))
            return rc;
    }
    const int base = c->hprm[inst].base;
    if (pressure && n) CK(cudaMemcpyAsync(pressure, c->d.press + base, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    if (youngs && n) CK(cudaMemcpyAsync(youngs, c->d.E + base, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CS3D_OK;
}

int cs3d_get_state_async(cs3d_ctx *c, int inst, int slot, int *n_cells, float *X, float *Y, float *Z, float *VX,
                         float *VY, float *VZ, float *pressure, float *youngs)
{
    if (!c || inst < 0 || inst >= c->n_inst || slot < 0 || slot > 1) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    int n = 0;
    if ((rc = inst_count(c, inst, &n))) return rc;
    if (n_cells) *n_cells = n;
    if (!c->copy_stream) CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    if (!c->astage[slot]) {
        // six node arrays and two per-cell arrays of the whole capacity
        const size_t words = (size_t)6 * c->cap_total * SLOTS + 2 * (size_t)c->cap_total;
        float *p = nullptr;
        if (cudaMalloc(&p, sizeof(float) * words) != cudaSuccess) return CS3D_E_NOMEM;
        c->allocs.push_back(p);
        c->astage[slot] = p;
        CK(cudaEventCreateWithFlags(&c->aready[slot], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->adone[slot], cudaEventDisableTiming));
    }
    if (n == 0) return CS3D_OK;
    float *stage = c->astage[slot];
    // the slot's previous copy must have left the staging buffer
    if (c->apending[slot]) CK(cudaStreamWaitEvent(c->stream, c->adone[slot], 0));
    const size_t k = (size_t)n * SLOTS;
    const size_t off = (size_t)c->hprm[inst].base * SLOTS;
    const int base = c->hprm[inst].base;
    const bool wx = X || Y || Z, wv = VX || VY || VZ;
    if (wx || wv)
        k_unpack<<<c->grid_flat, 256, 0, c->stream>>>(stage, wx ? (c->prekicked ? c->d.Xe : c->d.X) + off : nullptr,
                                                      wv ? (c->prekicked ? c->d.Vb : c->d.V) + off : nullptr, k);
    CK(cudaGetLastError());
    float *cellv = stage + 6 * k;
    if (pressure) CK(cudaMemcpyAsync(cellv, c->d.press + base, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
    if (youngs) CK(cudaMemcpyAsync(cellv + n, c->d.E + base, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaEventRecord(c->aready[slot], c->stream));
    CK(cudaStreamWaitEvent(c->copy_stream, c->aready[slot], 0));
    float *const out[6] = {X, Y, Z, VX, VY, VZ};
    for (int q = 0; q < 6; ++q)
        if (out[q]) CK(cudaMemcpyAsync(out[q], stage + (size_t)q * k, sizeof(float) * k, cudaMemcpyDeviceToHost,
                                       c->copy_stream));
    if (pressure) CK(cudaMemcpyAsync(pressure, cellv, sizeof(float) * n, cudaMemcpyDeviceToHost, c->copy_stream));
    if (youngs) CK(cudaMemcpyAsync(youngs, cellv + n, sizeof(float) * n, cudaMemcpyDeviceToHost, c->copy_stream));
    CK(cudaEventRecord(c->adone[slot], c->copy_stream));
    c->apending[slot] = true;
    return CS3D_OK;
}

int cs3d_wait_state(cs3d_ctx *c, int slot)
{
    if (!c || slot < 0 || slot > 1) return CS3D_E_ARG;
    if (!c->apending[slot]) return CS3D_OK;
    cudaSetDevice(c->device);
    CK(cudaEventSynchronize(c->adone[slot]));
    c->apending[slot] = false;
    return CS3D_OK;
}

int cs3d_host_alloc(size_t bytes, void **ptr)
{
    if (!ptr) return CS3D_E_ARG;
    *ptr = nullptr;
    if (cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) return CS3D_E_NOMEM;
    return CS3D_OK;
}

int cs3d_host_free(void *ptr)
{
    if (!ptr) return CS3D_OK;
    CK(cudaFreeHost(ptr));
    return CS3D_OK;
}

int cs3d_get_forces(cs3d_ctx *c, int inst, float *FCX, float *FCY, float *FCZ, float *FDX, float *FDY, float *FDZ)
{
    if (!c || inst < 0 || inst >= c->n_inst) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    int n = 0;
    if ((rc = inst_count(c, inst, &n))) return rc;
    float *const out[6] = {FCX, FCY, FCZ, FDX, FDY, FDZ};
    return fetch_soa(c, inst, n, (FCX || FCY || FCZ) ? c->d.FC : nullptr, (FDX || FDY || FDZ) ? c->d.FD : nullptr,
                     out);
}

int cs3d_get_random_force(cs3d_ctx *c, int inst, float *FRX, float *FRY, float *FRZ)
{
    if (!c || inst < 0 || inst >= c->n_inst) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    int n = 0;
    if ((rc = inst_count(c, inst, &n))) return rc;
    float *const out[6] = {FRX, FRY, FRZ, nullptr, nullptr, nullptr};
    return fetch_soa(c, inst, n, c->d.FR, nullptr, out);
}

int cs3d_get_cells(cs3d_ctx *c, int inst, float *cm, float *volume, float *area, float *aabb)
{
    if (!c || inst < 0 || inst >= c->n_inst) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    int n = 0;
    if ((rc = inst_count(c, inst, &n))) return rc;
    const int base = c->hprm[inst].base;
    if (cm && n) {
        std::vector<float4> b(n);
        CK(cudaMemcpyAsync(b.data(), c->d.CM + base, sizeof(float4) * n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int k = 0; k < n; ++k) { cm[3 * k] = b[k].x; cm[3 * k + 1] = b[k].y; cm[3 * k + 2] = b[k].z; }
    }
    if (volume && n) CK(cudaMemcpyAsync(volume, c->d.vol + base, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    if (area && n) CK(cudaMemcpyAsync(area, c->d.area + base, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    if (aabb && n) {
        std::vector<float4> b(2 * (size_t)n);
        int par = (int)(c->host_step & 1);
        CK(cudaMemcpyAsync(b.data(), c->d.aabb[par] + 2 * (size_t)base, sizeof(float4) * 2 * n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int k = 0; k < n; ++k) {
            const float4 lo = b[2 * k], hi = b[2 * k + 1];
            float *o = aabb + 6 * k;
            o[0] = lo.x; o[1] = hi.x; o[2] = lo.y; o[3] = hi.y; o[4] = lo.z; o[5] = hi.z;
        }
    }
    CK(cudaStreamSynchronize(c->stream));
    return CS3D_OK;
}

int cs3d_get_grid(cs3d_ctx *c, int inst, float minmax[6], int divs[3])
{
    if (!c || inst < 0 || inst >= c->n_inst) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    InstState st;
    CK(cudaMemcpyAsync(&st, &c->d.st[inst], sizeof st, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    int par = (int)(c->host_step & 1);
    for (int q = 0; q < 3; ++q) {
        auto dec = [](int i) { int b = i >= 0 ? i : i ^ 0x7fffffff; float f; memcpy(&f, &b, 4); return f; };
        float mn = std::min(dec(st.mm[par][2 * q]), 1.0e8f);
        float mx = std::max(dec(st.mm[par][2 * q + 1]), -1.0e8f);
        if (minmax) { minmax[2 * q] = mn; minmax[2 * q + 1] = mx; }
        volatile float ext = mx - mn;
        volatile float r = ext / DL;
        if (divs) divs[q] = (int)(r + 1.0f);
    }
    return CS3D_OK;
}

int cs3d_get_pairs(cs3d_ctx *c, int inst, int kind, int32_t *out, long long max_pairs, long long *count)
{
    if (!c || inst < 0 || inst >= c->n_inst || kind < 0 || kind > 1 || !count) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    unsigned long long np = 0;
    CK(cudaMemcpyAsync(&np, c->d.n_pairs, sizeof np, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if ((long long)np > c->d.pair_cap) return CS3D_E_CAPACITY;
    std::vector<int4> buf(np);
    if (np) CK(cudaMemcpyAsync(buf.data(), c->d.pairs, sizeof(int4) * np, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int base = c->hprm[inst].base, cap = c->hprm[inst].cap;
    long long k = 0;
    for (const int4 &p : buf) {
        int a = p.x >> 8, i = p.x & 255, b = p.y >> 8, j = p.y & 255;
        if (a < base || a >= base + cap) continue;
        bool keep = kind == 0 ? (p.z & 1) : 1;
        if (!keep) continue;
        if (out && k < max_pairs) {
            out[4 * k] = a - base; out[4 * k + 1] = i; out[4 * k + 2] = b - base; out[4 * k + 3] = j;
        }
        ++k;
    }
    *count = k;
    return CS3D_OK;
}

int cs3d_get_events(cs3d_ctx *c, int inst, int32_t *out, int max_events, int *count)
{
    if (!c || inst < 0 || inst >= c->n_inst || !count) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int ne = 0;
    CK(cudaMemcpyAsync(&ne, c->d.n_events, sizeof ne, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    ne = std::min(ne, c->d.ev_cap);
    std::vector<int4> buf(ne);
    if (ne) CK(cudaMemcpyAsync(buf.data(), c->d.events, sizeof(int4) * ne, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<int4> mine;
    for (auto &e : buf) if (e.x == inst) mine.push_back(e);
    std::sort(mine.begin(), mine.end(), [](const int4 &a, const int4 &b) {
        return a.y != b.y ? a.y < b.y : a.z < b.z;
    });
    int k = 0;
    for (auto &e : mine) {
        if (out && k < max_events) { out[3 * k] = e.y; out[3 * k + 1] = e.z; out[3 * k + 2] = e.w; }
        ++k;
    }
    *count = k;
    return CS3D_OK;
}

int cs3d_volume_histogram(cs3d_ctx *c, int inst, float lo, float hi, int nbins, int64_t *counts, float *volumes)
{
    if (!c || inst < 0 || inst >= c->n_inst || nbins < 1 || nbins > (1 << 20) || !counts || !(lo < hi) ||
        !std::isfinite(lo) || !std::isfinite(hi))
        return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int rc = ensure_init(c);
    if (rc) return rc;
    if ((rc = settle(c))) return rc;   // the volumes of the step-end positions
    int n = 0;
    if ((rc = inst_count(c, inst, &n))) return rc;
    // scratch for the counts and the volumes, freed before returning
    unsigned long long *dc = nullptr;
    float *dv = nullptr;
    if (cudaMalloc(&dc, sizeof(unsigned long long) * (nbins + 2)) != cudaSuccess) return CS3D_E_NOMEM;
    if (volumes && n && cudaMalloc(&dv, sizeof(float) * n) != cudaSuccess) { cudaFree(dc); return CS3D_E_NOMEM; }
    std::vector<unsigned long long> h(nbins + 2);
    cudaError_t e = cudaMemsetAsync(dc, 0, sizeof(unsigned long long) * (nbins + 2), c->stream);
    if (e == cudaSuccess && n) {
        const int blocks = std::min(n, c->nsm * 8);
        k_vol_hist<<<blocks, SLOTS, 0, c->stream>>>(c->d, inst, lo, hi, nbins, dc, dv);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), dc, sizeof(unsigned long long) * (nbins + 2), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && dv) e = cudaMemcpyAsync(volumes, dv, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(dc);
    if (dv) cudaFree(dv);
    if (e != cudaSuccess) return CS3D_E_CUDA;
    for (int b = 0; b < nbins + 2; ++b) counts[b] = (int64_t)h[b];
    return CS3D_OK;
}

int cs3d_get_far_counts(cs3d_ctx *c, int inst, int32_t *out, int max_entries, int *n_entries)
{
    if (!c || inst < 0 || inst >= c->n_inst || !n_entries) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    int nf = 0;
    CK(cudaMemcpyAsync(&nf, c->d.n_far, sizeof nf, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    nf = std::min(nf, c->d.far_cap);
    std::vector<int4> buf(nf);
    if (nf) CK(cudaMemcpyAsync(buf.data(), c->d.farlog, sizeof(int4) * nf, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<int4> mine;
    for (auto &e : buf) if (e.x == inst) mine.push_back(e);
    std::sort(mine.begin(), mine.end(), [](const int4 &a, const int4 &b) { return a.y < b.y; });
    int k = 0;
    for (auto &e : mine) {
        if (out && k < max_entries) { out[2 * k] = e.y; out[2 * k + 1] = e.z; }
        ++k;
    }
    *n_entries = k;
    return CS3D_OK;
}

int cs3d_last_error(cs3d_ctx *c, int inst, uint32_t *bits)
{
    if (!c || !bits || inst < -1 || inst >= c->n_inst) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    std::vector<InstState> st(c->n_inst);
    CK(cudaMemcpyAsync(st.data(), c->d.st, sizeof(InstState) * c->n_inst, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    unsigned b = 0;
    for (int k = 0; k < c->n_inst; ++k)
        if (inst < 0 || k == inst) b |= st[k].err;
    *bits = b;
    return CS3D_OK;
}

int cs3d_get_stats(cs3d_ctx *c, long long *stats, int n)
{
    if (!c || !stats || n <= 0) return CS3D_E_ARG;
    cudaSetDevice(c->device);
    std::vector<InstState> st(c->n_inst);
    CK(cudaMemcpyAsync(st.data(), c->d.st, sizeof(InstState) * c->n_inst, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    long long v[8] = {c->host_step, 0, 0, 0, c->launches_per_step, 0, 0, 0};
    for (auto &q : st) v[5] = std::max<long long>(v[5], q.max_halo);
    for (auto &q : st) {
        v[1] += q.rebuilds;
        v[2] = std::max<long long>(v[2], q.max_entries);
        v[3] = std::max<long long>(v[3], q.max_cand);
        v[6] += q.built;
        v[7] += q.rebuilds_div;
    }
    for (int k = 0; k < n && k < 8; ++k) stats[k] = v[k];
    return CS3D_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// cs3d_forces_static: the initial force evaluation on caller-owned device
// buffers, with every scratch buffer carved out of one file-scope static
// device array (no allocation anywhere on this path).
// ---------------------------------------------------------------------------
namespace {

constexpr int SCAP = CS3D_STATIC_MAX_CELLS;
constexpr int SHASH = hash_size(2 * SCAP);   // bucket rule of cs3d_create_ensemble
constexpr int SEVENTS = 16;

struct StaticScratch {
    InstParams prm;
    InstState st;
    float4 X[SCAP * SLOTS], V[SCAP * SLOTS], Vb[SCAP * SLOTS], FC[SCAP * SLOTS], FD[SCAP * SLOTS], Xb[SCAP * SLOTS];
    float4 FR[SCAP * SLOTS];
    float4 CM[SCAP];
    float press[SCAP], E[SCAP], vol[SCAP], area[SCAP];
    uint8_t divflag[SCAP];
    float4 aabb0[2 * SCAP], aabb1[2 * SCAP];
    float4 hpos[SCAP * SLOTS];
    alignas(16) int hcount[SHASH + SCAN_TILE];
    int hscan[SHASH / SCAN_TILE + 1], node_rank[SCAP * SLOTS], hsz;
    int cell_inst[SCAP], work[SCAP], work_n;
    int cand[SCAP * MAXC], ncand[SCAP];
    uint16_t dlist[SCAP * MAXD * SLOTS];
    uint8_t ndis[SCAP * SLOTS];
    int dirty[SCAP];
    uint16_t ent[SCAP * MAXE * SLOTS];
    uint8_t nent[SCAP * SLOTS];
    DivEntry divtab[SCAP];
    int div_total;
    int4 events[SEVENTS];
    int n_events;
    int flags[4];
    int4 pairs[1];
    unsigned long long n_pairs;
    uint32_t nnpack[SLOTS];
    float4 r0[SLOTS], th0[SLOTS];
    uint4 arm[SLOTS];
    uint8_t faces[CS3D_FACES * 7];
    double2 cs0[3 * SLOTS];
    double r0i[3 * SLOTS];
};

// The scratch of cs3d_forces_static.  In host code this name is only a
// stand-in for the device object: kernels receive the address resolved with
// cudaGetSymbolAddress, per device.
static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

struct StaticDevice {
    bool ready = false;
    StaticScratch *base = nullptr;
    int grid_cells = 1, grid_flat = 1, grid_nodes = 1, grid_tiles = 1;
};

constexpr int kMaxDevices = 64;
StaticDevice g_static_dev[kMaxDevices];
std::mutex g_static_mutex;

Dev static_dev(StaticScratch *s)
{
    Dev d{};
    d.n_inst = 1;
    d.cap_total = SCAP;
    d.single = 1;
    d.prm = &s->prm;
    d.st = &s->st;
    d.topo.nnpack = s->nnpack;
    d.topo.r0 = s->r0;
    d.topo.th0 = s->th0;
    d.topo.arm = s->arm;
    d.topo.faces = s->faces;
    d.topo.cs0 = s->cs0;
    d.topo.r0i = s->r0i;
    d.X = s->X; d.V = s->V; d.Vb = s->Vb; d.FC = s->FC; d.FD = s->FD; d.Xb = s->Xb; d.FR = s->FR;
    d.CM = s->CM;
    d.press = s->press; d.E = s->E; d.vol = s->vol; d.area = s->area;
    d.divflag = s->divflag;
    d.aabb[0] = s->aabb0; d.aabb[1] = s->aabb1;
    d.cell_inst = s->cell_inst; d.work = s->work; d.work_n = &s->work_n;
    d.cand = s->cand; d.ncand = s->ncand;
    d.dlist = s->dlist; d.ndis = s->ndis; d.dirty = s->dirty;
    d.ent = s->ent; d.nent = s->nent;
    d.hsize = SHASH; d.hsz = &s->hsz; d.hcount = s->hcount; d.hscan = s->hscan; d.hpos = s->hpos; d.node_rank = s->node_rank;
    d.divtab = s->divtab; d.div_total = &s->div_total;
    d.events = s->events; d.n_events = &s->n_events; d.ev_cap = SEVENTS;
    d.flags = s->flags;
    d.pairs = s->pairs; d.n_pairs = &s->n_pairs; d.pair_cap = 1; d.record_pairs = 0;
    return d;
}

// Caller's 192-stride SoA inputs into the scratch (float4), defaults for the
// per-cell arrays, zero forces.
__global__ void k_static_load(Dev d, int n, const float *X, const float *Y, const float *Z, const float *VX,
                              const float *VY, const float *VZ, const float *press, const float *E, float minp,
                              float stiff1)
{
    const int total = n * SLOTS;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const bool real = (g % SLOTS) < NODES;
        d.X[g] = real ? make_float4(X[g], Y[g], Z[g], 0.f) : make_float4(0, 0, 0, 0);
        d.V[g] = (real && VX) ? make_float4(VX[g], VY[g], VZ[g], 0.f) : make_float4(0, 0, 0, 0);
        d.FC[g] = make_float4(0, 0, 0, 0);
        d.FD[g] = make_float4(0, 0, 0, 0);
        if (g < n) {
            d.press[g] = press ? press[g] : minp;
            d.E[g] = E ? E[g] : stiff1;
            d.cell_inst[g] = 0;
            d.CM[g] = make_float4(0, 0, 0, 0);
        }
    }
}

__global__ void k_static_store(Dev d, int n, float *FCX, float *FCY, float *FCZ, float *FDX, float *FDY, float *FDZ)
{
    const int total = n * SLOTS;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const bool real = (g % SLOTS) < NODES;
        const float4 c = real ? d.FC[g] : make_float4(0, 0, 0, 0);
        const float4 f = real ? d.FD[g] : make_float4(0, 0, 0, 0);
        FCX[g] = c.x; FCY[g] = c.y; FCZ[g] = c.z;
        FDX[g] = f.x; FDY[g] = f.y; FDZ[g] = f.z;
    }
}

// Per-device set-up: resolve the static array's device address and set the
// kernel attributes the init sequence needs.  Runs once per device and keeps
// the address for the life of the process: a cudaDeviceReset (or any other
// teardown of the device's primary context) invalidates it, and the entry
// point must not be called on that device afterwards.
int static_setup(int dev, StaticDevice **out)
{
    if (dev < 0 || dev >= kMaxDevices) return CS3D_E_ARG;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    StaticDevice &sd = g_static_dev[dev];
    if (!sd.ready) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr) {
            fprintf(stderr, "cs3d: cudaGetSymbolAddress of the static scratch failed: %s\n", cudaGetErrorString(e));
            return CS3D_E_CUDA;
        }
        sd.base = (StaticScratch *)ptr;
        CK(cudaFuncSetAttribute(k_s1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(S1Smem)));
        int nsm = 148, occ = 1;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_s1<true>, SLOTS, sizeof(S1Smem)));
        sd.grid_cells = std::max(1, std::min(SCAP, nsm * std::max(occ, 1)));
        sd.grid_flat = std::max(1, std::min((SCAP * SLOTS + 255) / 256, nsm * 8));
        sd.grid_nodes = std::max(1, std::min(SCAP, nsm * 8));
        sd.grid_tiles = std::max(1, std::min(SHASH / SCAN_TILE + 1, nsm * 8));
        sd.ready = true;
    }
    *out = &sd;
    return CS3D_OK;
}

}  // namespace

extern "C" int cs3d_forces_static(const cs3d_params *params, const cs3d_topology *topo, int n_cells,
                                  const float *X, const float *Y, const float *Z, const float *VX, const float *VY,
                                  const float *VZ, const float *pressure, const float *youngs, float *FCX,
                                  float *FCY, float *FCZ, float *FDX, float *FDY, float *FDZ, void *stream)
{
    if (!params || !topo || !X || !Y || !Z || !FCX || !FCY || !FCZ || !FDX || !FDY || !FDZ) return CS3D_E_ARG;
    if ((VX || VY || VZ) && !(VX && VY && VZ)) return CS3D_E_ARG;
    if (n_cells < 1 || n_cells > SCAP) {
        fprintf(stderr, "cs3d_forces_static: %d cells requested, the static scratch holds 1..%d\n", n_cells, SCAP);
        return CS3D_E_ARG;
    }
    if (check_params(*params)) return CS3D_E_CONFIG;
    TopoTables tt;
    int rc = topo_tables(topo, tt);
    if (rc) return rc;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    StaticDevice *sd = nullptr;
    if ((rc = static_setup(dev, &sd))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    StaticScratch *S = sd->base;
    const Dev d = static_dev(S);
    // parameters, mesh tables and a cleared instance state
    const InstParams ip = make_inst(*params, 0, SCAP, 0.1f);
    InstState st0;
    memset(&st0, 0, sizeof st0);
    st0.n = n_cells;
    CK(cudaMemcpyAsync(&S->prm, &ip, sizeof ip, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(&S->st, &st0, sizeof st0, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S->nnpack, tt.nnp, sizeof tt.nnp, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S->r0, tt.r0, sizeof tt.r0, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S->th0, tt.th, sizeof tt.th, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S->arm, tt.arm, sizeof tt.arm, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S->faces, tt.faces, sizeof tt.faces, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S->cs0, tt.cs0, sizeof tt.cs0, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S->r0i, tt.r0i, sizeof tt.r0i, cudaMemcpyHostToDevice, s));
    // the previous call's neighbour lists, boxes and flags must not leak in
    CK(cudaMemsetAsync(S->ncand, 0, sizeof S->ncand, s));
    CK(cudaMemsetAsync(S->nent, 0, sizeof S->nent, s));
    CK(cudaMemsetAsync(S->dirty, 0, sizeof S->dirty, s));
    CK(cudaMemsetAsync(S->flags, 0, sizeof S->flags, s));
    CK(cudaMemsetAsync(&S->n_events, 0, sizeof S->n_events, s));
    k_static_load<<<sd->grid_flat, 256, 0, s>>>(d, n_cells, X, Y, Z, VX, VY, VZ, pressure, youngs, params->min_pressure,
                                                  params->stiffness1);
    // the initialisation sequence of run_init on the static buffers
    k_build_work<<<1, 256, 0, s>>>(d);
    k_init_begin<<<1, 256, 0, s>>>(d);
    k_geom<<<sd->grid_cells, SLOTS, 0, s>>>(d, 0);
    // correct_com at set-up, as run_init (src/GPUbounce.cu:785-805): the shift
    // moves the positions the wall and contact forces see
    if (params->correct_com) k_com_shift<<<1, 256, 0, s>>>(d);
    if ((rc = launch_nl_kernels(d, s, sd->grid_nodes, sd->grid_tiles))) return rc;
    k_s1<true><<<sd->grid_cells, SLOTS, sizeof(S1Smem), s>>>(d, 0);
    k_static_store<<<sd->grid_flat, 256, 0, s>>>(d, n_cells, FCX, FCY, FCZ, FDX, FDY, FDZ);
    CK(cudaGetLastError());
    unsigned err = 0;
    CK(cudaMemcpyAsync(&err, &S->st.err, sizeof err, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return err ? CS3D_E_DEVICE_FLAGS : CS3D_OK;
}
