// cs3d_main.cpp -- command-line driver, a drop-in for the reference's
// CellDiv executable (src/GPUbounce.cu:267-1594):
//
//     cs3d <no_of_cells> <inp.json> <gpu_id>
//
// Reads the same inp.json and mesh files (C180, C180NN, C180C,
// C180_pentahexa from the working directory), places the cells as
// initialize_C180s does, runs div_time_steps + non_div_time_steps steps on
// the GPU through libcs3d.so and writes the same binary (or ASCII)
// trajectory and mitotic-index file.
//
// Extension: if the environment variable CS3D_INIT_FILE names a file, the
// initial state is read from it instead of being placed (format: the 8 bytes
// "CS3DINIT", int32 n, then float32 X, Y, Z, VX, VY, VZ [n*192 each],
// pressure [n], youngs [n]).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cs3d.h"

namespace {

int fail(const char *what, int rc)
{
    fprintf(stderr, "cs3d: %s: %s (%d)\n", what, cs3d_strerror(rc), rc);
    return rc == 0 ? 1 : rc;
}

bool read_init_file(const char *path, int &n, std::vector<float> &a, std::vector<float> &pv,
                    std::vector<float> &ev)
{
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    char magic[8];
    int32_t nn = 0;
    bool ok = fread(magic, 1, 8, f) == 8 && !memcmp(magic, "CS3DINIT", 8) && fread(&nn, 4, 1, f) == 1 && nn > 0;
    if (ok) {
        n = nn;
        size_t k = (size_t)n * 192;
        a.assign(6 * k, 0.f);
        pv.assign(n, 0.f);
        ev.assign(n, 0.f);
        ok = fread(a.data(), 4, 6 * k, f) == 6 * k && fread(pv.data(), 4, n, f) == (size_t)n &&
             fread(ev.data(), 4, n, f) == (size_t)n;
    }
    fclose(f);
    return ok;
}

// Stiffness class of every cell for the trajectory: 0 (stiffness1) or 1,
// src/GPUbounce.cu:2459-2464.
void cell_types(const cs3d_params &p, int n, const float *E, std::vector<int32_t> &t)
{
    t.resize(n > 0 ? n : 1);
    for (int c = 0; c < n; ++c) t[c] = E[c] == p.stiffness1 ? 0 : 1;
}

void write_ascii_frame(FILE *f, int step, int interval, int n, const float *X, const float *Y, const float *Z,
                       const cs3d_params &prm, const float *E)
{
    // write_traj, src/GPUbounce.cu:2412-2444 (cell labels H / C with variable stiffness)
    fprintf(f, "%d\n", n * 192);
    fprintf(f, "Step: %d frame: %d\n", step, step / interval);
    for (int c = 0; c < n; c++) {
        if (!prm.use_different_stiffnesses) fprintf(f, "cell: %d\n", c);
        else if (E[c] == prm.stiffness1) fprintf(f, "cell: %d H\n", c);
        else if (E[c] == prm.stiffness2) fprintf(f, "cell: %d C\n", c);
        else fprintf(f, "cell: %d UnknownStiffness\n", c);
        for (int p = 0; p < 192; p++)
            fprintf(f, "%.7f,  %.7f,  %.7f\n", X[c * 192 + p], Y[c * 192 + p], Z[c * 192 + p]);
    }
}

// writeForces, src/GPUbounce.cu:2567-2597: one line per node with the total
// conservative force, the velocity, the position, and the cell's pressure and
// volume (the volume of the last division test; 0 before any).
void write_force_rows(FILE *f, int step, int n, const float *FX, const float *FY, const float *FZ, const float *VX,
                      const float *VY, const float *VZ, const float *X, const float *Y, const float *Z,
                      const float *press, const float *vol)
{
    auto mag = [](float x, float y, float z) { return sqrtf(x * x + y * y + z * z); };
    for (int c = 0; c < n; ++c)
        for (int k = 0; k < 180; ++k) {
            const size_t g = (size_t)c * 192 + k;
            fprintf(f, "%d,%d,%d,%d,%d,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f,%.8f\n", step, n, c, k,
                    (int)g, FX[g], FY[g], FZ[g], mag(FX[g], FY[g], FZ[g]), VX[g], VY[g], VZ[g],
                    mag(VX[g], VY[g], VZ[g]), X[g], Y[g], Z[g], press[c], vol[c]);
        }
}

// The force file of write_cont_force: the state of the device at a frame.
int write_forces_frame(cs3d_ctx *ctx, FILE *f, int step, size_t cap_nodes, int max_cells, const float *X0,
                       const float *Y0, const float *Z0)
{
    std::vector<float> F[3], V[3], P[3], press(max_cells), vol(max_cells);
    for (int q = 0; q < 3; ++q) {
        F[q].assign(cap_nodes, 0.f);
        V[q].assign(cap_nodes, 0.f);
        if (!X0) P[q].assign(cap_nodes, 0.f);
    }
    int n = 0, rc;
    if ((rc = cs3d_get_state(ctx, 0, &n, X0 ? nullptr : P[0].data(), X0 ? nullptr : P[1].data(),
                             X0 ? nullptr : P[2].data(), V[0].data(), V[1].data(), V[2].data(), press.data(), nullptr)))
        return rc;
    if ((rc = cs3d_get_forces(ctx, 0, F[0].data(), F[1].data(), F[2].data(), nullptr, nullptr, nullptr))) return rc;
    if ((rc = cs3d_get_cells(ctx, 0, nullptr, vol.data(), nullptr, nullptr))) return rc;
    write_force_rows(f, step, n, F[0].data(), F[1].data(), F[2].data(), V[0].data(), V[1].data(), V[2].data(),
                     X0 ? X0 : P[0].data(), X0 ? Y0 : P[1].data(), X0 ? Z0 : P[2].data(), press.data(), vol.data());
    return CS3D_OK;
}

}  // namespace

int main(int argc, char **argv)
{
    printf("cs3d (CellSim3D timestep on B200) version %d\n", cs3d_version());
    if (argc != 4) {
        printf("Usage: cs3d no_of_cells inpFile.json gpuid\n");
        return 0;
    }
    int n0 = atoi(argv[1]);
    int gpu = atoi(argv[3]);
    cs3d_config cfg;
    char err[512] = {0};
    int rc = cs3d_config_read_json(argv[2], &cfg, err, sizeof err);
    if (rc) {
        fprintf(stderr, "%s\n", err);
        return -1;
    }
    if (n0 > cfg.max_cells || n0 < 0) {
        printf("no_of_cells should be < %d\n", cfg.max_cells);
        return 0;
    }
    cs3d_params prm;
    rc = cs3d_config_to_params(&cfg, &prm);
    if (rc) return fail("unsupported or invalid parameters in inp.json", rc);
    // RNG seeds, src/GPUbounce.cu:1777-1810
    if (cfg.rand_seed < 0) {
        time_t now = time(nullptr);
        prm.rng_ij = (int)(now % 31328);
        prm.rng_kl = (int)(now % 30081);
    }
    cs3d_rng rng;
    if ((rc = cs3d_rng_init(&rng, prm.rng_ij, prm.rng_kl))) return fail("RNG seeds", rc);
    printf("RNG seeds: %d, %d\n", prm.rng_ij, prm.rng_kl);
    cs3d_mesh mesh;
    if ((rc = cs3d_mesh_read(".", &mesh))) return fail("reading C180, C180NN, C180C, C180_pentahexa", rc);
    const size_t cap_nodes = (size_t)cfg.max_cells * 192;
    std::vector<float> X(cap_nodes, 0.f), Y(cap_nodes, 0.f), Z(cap_nodes, 0.f);
    std::vector<float> VX, VY, VZ, press, youngs;
    const char *init_file = getenv("CS3D_INIT_FILE");
    if (init_file && *init_file) {
        std::vector<float> a;
        int n = 0;
        if (!read_init_file(init_file, n, a, press, youngs) || n > cfg.max_cells) return fail("CS3D_INIT_FILE", CS3D_E_IO);
        n0 = n;
        size_t k = (size_t)n * 192;
        std::copy(a.begin(), a.begin() + k, X.begin());
        std::copy(a.begin() + k, a.begin() + 2 * k, Y.begin());
        std::copy(a.begin() + 2 * k, a.begin() + 3 * k, Z.begin());
        VX.assign(a.begin() + 3 * k, a.begin() + 4 * k);
        VY.assign(a.begin() + 4 * k, a.begin() + 5 * k);
        VZ.assign(a.begin() + 5 * k, a.begin() + 6 * k);
    } else {
        if ((rc = cs3d_init_positions(&cfg, &mesh, n0, &rng, X.data(), Y.data(), Z.data())))
            return fail("initial placement", rc);
    }
    if (youngs.empty()) {
        // softer cells at set-up, src/GPUbounce.cu:616-692
        youngs.assign(cfg.max_cells, 0.f);
        if ((rc = cs3d_initial_stiffness(&cfg, n0, X.data(), Y.data(), Z.data(), &rng, youngs.data()))) {
            if (rc == CS3D_E_CONFIG) printf("ERROR: Too many softer cells requested\n");
            return fail("initial stiffness", rc);
        }
    }
    cs3d_topology topo;
    if ((rc = cs3d_topology_build(&mesh, X.data(), Y.data(), Z.data(), &topo))) return fail("mesh tables", rc);
    cs3d_ctx *ctx = nullptr;
    if ((rc = cs3d_create(&prm, &topo, cfg.max_cells, gpu, nullptr, &ctx))) return fail("device context", rc);
    rc = cs3d_load_state(ctx, 0, n0, X.data(), Y.data(), Z.data(), VX.empty() ? nullptr : VX.data(),
                         VY.empty() ? nullptr : VY.data(), VZ.empty() ? nullptr : VZ.data(),
                         press.empty() ? nullptr : press.data(), youngs.empty() ? nullptr : youngs.data());
    if (rc) return fail("loading the initial state", rc);
    if ((rc = cs3d_set_rng(ctx, 0, &rng))) return fail("RNG state", rc);

    const int total_steps = cfg.div_time_steps + cfg.non_div_time_steps;
    const int interval = cfg.traj_write_int;
    FILE *ascii = nullptr;
    cs3d_traj *traj = nullptr;
    const int max_frames = (total_steps + 1) / interval;
    const int varstiff = cfg.use_different_stiffnesses ? 1 : 0;
    if (cfg.binary_output) {
        if ((rc = cs3d_traj_open(cfg.traj_file_name, cfg.max_cells, varstiff, max_frames, &traj)))
            return fail("trajectory file", rc);
        std::vector<int32_t> types;
        cell_types(prm, n0, youngs.data(), types);
        if ((rc = cs3d_traj_write_frame(traj, 0, 1, n0, X.data(), Y.data(), Z.data(), types.data())))
            return fail("trajectory frame", rc);
    } else {
        ascii = fopen(cfg.traj_file_name, "w");
        if (!ascii) return fail("trajectory file", CS3D_E_IO);
        fprintf(ascii, "Header Start:\nMaximum number of cells:\n%d\nUsing variable stiffness:\n%s\n"
                       "Maximum number of frames:\n%d\nHeader End\n", cfg.max_cells, varstiff ? "True" : "False",
                max_frames);
        write_ascii_frame(ascii, 0, interval, n0, X.data(), Y.data(), Z.data(), prm, youngs.data());
    }
    // force file, src/GPUbounce.cu:1030-1047 (header and the initial forces;
    // the positions are the host's initial ones, as there)
    FILE *forces = nullptr;
    if (cfg.write_cont_force) {
        forces = fopen(cfg.forces_file, "w");
        if (!forces) return fail("forces file", CS3D_E_IO);
        fprintf(forces, "step,num_cells,cell_ind,node_ind,glob_node_ind,FX,FY,FZ,F,VX,VY,VZ,V,X,Y,Z,P,Vol\n");
        if ((rc = write_forces_frame(ctx, forces, 0, cap_nodes, cfg.max_cells, X.data(), Y.data(), Z.data())))
            return fail("forces file", rc);
    }
    int frame = 1;
    int step = 0;
    int n = n0;
    // Frames are read back asynchronously into one of two page-locked host
    // buffers (cs3d_get_state_async: the device-to-host copy runs on a copy
    // stream while the GPU steps on) and written by a second thread (the
    // reference reads and writes them on the step loop's thread while the GPU
    // idles, src/GPUbounce.cu:1430-1475).  Frame k is copied into buffer
    // k % 2; when frame k + 1 is due, frame k's copy has long landed: it is
    // handed to the writer thread, and buffer (k + 1) % 2 is free once the
    // writer of frame k - 1 has finished.
    float *WB[2][4] = {};   // X, Y, Z per node, stiffness per cell
    for (auto &b : WB)
        for (int q = 0; q < 4; ++q)
            if ((rc = cs3d_host_alloc(sizeof(float) * (q < 3 ? cap_nodes : (size_t)cfg.max_cells), (void **)&b[q])))
                return fail("page-locked frame buffers", rc);
    auto free_buffers = [&]() {
        cs3d_wait_state(ctx, 0);
        cs3d_wait_state(ctx, 1);
        for (auto &b : WB)
            for (float *&p : b) { cs3d_host_free(p); p = nullptr; }
    };
    std::thread writer;
    int wrc = 0;
    auto join_writer = [&]() {
        if (writer.joinable()) writer.join();
        return wrc;
    };
    struct Pending { bool valid; int slot, step, frame, n; } pend = {false, 0, 0, 0, 0};
    // hand the pending frame (its copy finished) to the writer thread
    auto write_pending = [&]() -> int {
        if (!pend.valid) return 0;
        int r = cs3d_wait_state(ctx, pend.slot);
        if (r) return r;
        if (join_writer()) return wrc;
        float *const *b = WB[pend.slot];
        const Pending p = pend;
        writer = std::thread([&wrc, &prm, traj, ascii, b, p, interval]() {
            if (traj) {
                std::vector<int32_t> types;
                cell_types(prm, p.n, b[3], types);
                wrc = cs3d_traj_write_frame(traj, p.step, p.frame, p.n, b[0], b[1], b[2], types.data());
            } else {
                write_ascii_frame(ascii, p.step, interval, p.n, b[0], b[1], b[2], prm, b[3]);
            }
        });
        pend.valid = false;
        return 0;
    };
    int slot = 0;
    while (step < total_steps) {
        int chunk = interval - step % interval;
        if (step + chunk > total_steps) chunk = total_steps - step;
        rc = cs3d_step(ctx, chunk);
        step += chunk;
        if (rc) {
            join_writer();
            free_buffers();
            uint32_t bits = 0;
            cs3d_last_error(ctx, 0, &bits);
            fprintf(stderr, "cs3d: step %d: %s (error bits 0x%x)\n", step, cs3d_strerror(rc), bits);
            if (rc == CS3D_E_CAPACITY) {
                printf("ERROR: Population exceeded the %d allocated cells\n", cfg.max_cells);
                return -69;
            }
            return -1;
        }
        if (step % 1000 < chunk || chunk >= 1000) {
            cs3d_get_state(ctx, 0, &n, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
            printf("   time %-8d %d cells\n", step, n);
        }
        if (step % interval == 0) {
            ++frame;
            // the previous frame to the writer; its thread then owns that
            // buffer, and this frame's buffer is free (its writer joined)
            if ((rc = write_pending())) {
                join_writer();
                free_buffers();
                return fail("trajectory frame", rc);
            }
            float *const *b = WB[slot];
            if ((rc = cs3d_get_state_async(ctx, 0, slot, &n, b[0], b[1], b[2], nullptr, nullptr, nullptr, nullptr,
                                           b[3]))) {
                join_writer();
                free_buffers();
                return fail("reading the state", rc);
            }
            pend = {true, slot, step, frame, n};
            slot ^= 1;
            // forces at the frame, src/GPUbounce.cu:1455-1473
            if (forces && (rc = write_forces_frame(ctx, forces, step, cap_nodes, cfg.max_cells, nullptr, nullptr,
                                                   nullptr))) {
                join_writer();
                free_buffers();
                return fail("forces file", rc);
            }
        }
    }
    if ((rc = write_pending())) {
        join_writer();
        free_buffers();
        return fail("trajectory frame", rc);
    }
    if (forces) fclose(forces);
    if (join_writer()) {
        free_buffers();
        return fail("trajectory frame", wrc);
    }
    free_buffers();
    cs3d_get_state(ctx, 0, &n, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (traj) cs3d_traj_close(traj, n);
    if (ascii) fclose(ascii);
    float mm[6];
    int divs[3];
    cs3d_get_grid(ctx, 0, mm, divs);
    printf("Xdiv = %d, Ydiv = %d, Zdiv = %d\n", divs[0], divs[1], divs[2]);

    // mitotic index file, src/GPUbounce.cu:1288-1302 and :1515-1547; with
    // count_only_internal_cells the far daughters of a step are not counted
    // (num_cells_far, :2538-2565)
    int nev = 0;
    cs3d_get_events(ctx, 0, nullptr, 0, &nev);
    std::vector<int32_t> ev(3 * (size_t)(nev > 0 ? nev : 1));
    cs3d_get_events(ctx, 0, ev.data(), nev, &nev);
    int nfar = 0;
    cs3d_get_far_counts(ctx, 0, nullptr, 0, &nfar);
    std::vector<int32_t> far(2 * (size_t)(nfar > 0 ? nfar : 1));
    cs3d_get_far_counts(ctx, 0, far.data(), nfar, &nfar);
    const int cci = cfg.cell_count_int;
    const int nbuckets = cfg.div_time_steps / cci + 1;
    std::vector<int> born(cfg.div_time_steps + 2, 0), per_step(cfg.div_time_steps + 2, 0);
    for (int k = 0; k < nev; ++k)
        if (ev[3 * k] >= 1 && ev[3 * k] <= cfg.div_time_steps) born[ev[3 * k]] += 1;
    per_step = born;
    for (int k = 0; k < nfar; ++k)
        if (far[2 * k] >= 1 && far[2 * k] <= cfg.div_time_steps) per_step[far[2 * k]] -= far[2 * k + 1];
    std::vector<int> dividing(nbuckets, 0), totals(nbuckets, 0);
    int cells = n0;
    for (int s = 1; s <= cfg.div_time_steps; ++s) {
        cells += born[s];
        if (s % cci == 0) {
            int nc = 0;
            for (int q = 0; q < cci; ++q) nc += per_step[s - cci + 1 + q];
            dividing[(s - 1) / cci] = nc;
            totals[(s - 1) / cci] = cells - nc;
        }
    }
    FILE *mi = fopen(cfg.mit_index_file, cfg.overwrite_mit_ind ? "w" : "a");
    if (mi) {
        for (int q = 0; q < nbuckets; ++q)
            fprintf(mi, "%f\n", (dividing[q] != 0 && totals[q] != 0) ? (float)dividing[q] / totals[q] : 0.0);
        fclose(mi);
    }
    cs3d_destroy(ctx);
    return 0;
}
