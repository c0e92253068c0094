/*
 * cs3d.h -- C ABI of libcs3d.so, the B200-native timestep of CellSim3D.
 *
 * Every function returns an int status: 0 = success, negative = CS3D_E_*.
 * No C++ exceptions and no torch types cross this boundary; all buffers are
 * plain pointers with explicit sizes.  Host arrays are caller-owned and are
 * copied synchronously on the context's stream.  A context owns all of its
 * device memory and is used by one host thread at a time.
 *
 * Layout conventions follow the reference (SoftSimu/CellSim3D):
 *   - per-node arrays are SoA float, indexed cell*192 + node for nodes
 *     0..179 (slots 180..191 are padding), src/GPUbounce.cu:365-373;
 *   - per-cell arrays are indexed by cell;
 *   - neighbour tables are [k*192 + node], src/GPUbounce.cu:1829-1832.
 */
#ifndef CS3D_H
#define CS3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS3D_SLOTS 192
#define CS3D_NODES 180
#define CS3D_FACES 92

/* ---- status codes ----------------------------------------------------- */
#define CS3D_OK                 0
#define CS3D_E_ARG             -1   /* invalid argument / size */
#define CS3D_E_CUDA            -2   /* a CUDA runtime call failed */
#define CS3D_E_NOMEM           -3   /* device or host allocation failed */
#define CS3D_E_IO              -4   /* file could not be opened / read */
#define CS3D_E_PARSE           -5   /* inp.json malformed or missing section */
#define CS3D_E_CONFIG          -6   /* parameter validation failed */
#define CS3D_E_DEVICE_FLAGS    -7   /* a kernel raised an error bit, see cs3d_last_error */
#define CS3D_E_CAPACITY       -69   /* population exceeded capacity, src/GPUbounce.cu:1265-1270; as in the
                                       reference (which exits), the run ends there: the cells that could
                                       not divide did not take the step's last half kick either */
#define CS3D_E_UNSUPPORTED     -8   /* feature of the reference outside this library */

/* ---- device error bits (cs3d_last_error) ------------------------------ */
#define CS3D_ERRBIT_NAN            0x001u  /* NaN position, src/propagate.cu:241-248 */
#define CS3D_ERRBIT_CAPACITY       0x002u  /* division past capacity */
#define CS3D_ERRBIT_CAND_OVERFLOW  0x004u  /* > CS3D_MAX_CAND contact cells for one cell */
#define CS3D_ERRBIT_ENTRY_OVERFLOW 0x008u  /* > CS3D_MAX_ENTRIES contact nodes or > CS3D_MAX_DIS pairs for one node */
#define CS3D_ERRBIT_NONFINITE_VOL  0x010u  /* src/volume.cu:134-139 */
#define CS3D_ERRBIT_BAD_NORMAL     0x020u  /* |n| != 1, src/postscriptinit.cu:215-219 */
#define CS3D_ERRBIT_GRID_OVERFLOW  0x040u  /* reserved, never raised (the node hash cannot overflow) */
#define CS3D_ERRBIT_PAIR_OVERFLOW  0x080u  /* pair-recording buffer full */
#define CS3D_ERRBIT_HALO_OVERFLOW  0x100u  /* reserved, never raised */
#define CS3D_ERRBIT_SOFT_CELLS     0x200u  /* more distinct softer cells requested than cell indices
                                              exist (the reference loops forever, src/GPUbounce.cu:1364-1384) */

#define CS3D_MAX_CAND     128   /* contact-candidate cells per cell */
#define CS3D_MAX_ENTRIES   64   /* contact-candidate nodes per node */
#define CS3D_MAX_DIS       32   /* dissipative contact pairs per node and step */

/* ---- parameters of the hot path (one simulation instance) ------------- */
/* Field meaning and units are the reference's inp.json keys.              */
typedef struct cs3d_params {
    float particle_mass;        /* core.particle_mass */
    float repulsion_range;      /* core.repulsion_range */
    float attraction_range;     /* core.attraction_range */
    float repulsion_strength;   /* core.repulsion_strength (x Youngs_mod) */
    float attraction_strength;  /* core.attraction_strength (x Youngs_mod) */
    float youngs_mod;           /* core.Youngs_mod */
    float stiffness1;           /* core.stiffFactor1 * Youngs_mod, src/GPUbounce.cu:1953 */
    float internal_damping;     /* core.internal_damping (gamma_int) */
    float viscotic_damping;     /* core.viscotic_damping (gamma_ext) */
    float gamma_visc;           /* core.gamma_visc (gamma_o) */
    float division_vol;         /* core.division_Vol */
    float time_interval;        /* core.time_interval */
    float max_pressure;         /* core.maxPressure */
    float min_pressure;         /* core.minPressure */
    float growth_rate;          /* core.growth_rate (rMax; no population model) */
    float thresh_dist;          /* walls.threshDist */
    float box_len[3];           /* boxParams.box_len_{x,y,z} = boxMax */
    int32_t check_sphericity;   /* core.checkSphericity */
    int32_t constrain_angles;   /* core.constrainAngles */
    int32_t use_rigid_box;      /* boxParams.useRigidSimulationBox */
    int32_t daught_same_stiffness; /* stiffnessParams.daughtSameStiffness */
    int32_t div_time_steps;     /* core.div_time_steps */
    int32_t rng_ij, rng_kl;     /* RANMAR seeds (see cs3d_seed_map) */
    /* Langevin random force (rand_params.add_rands, src/propagate.cu:668-678):
     * per node and step rand_scale_factor times three standard normals, used
     * in VelocityUpdateA and the next Integrate with weight sqrt(dt).  The
     * reference draws them from curand XORWOW states; this library draws them
     * from Philox4x32-10 keyed by rand_seed and counted by (node, step), so
     * only their distribution, not their values, matches the reference. */
    int32_t add_rands;          /* rand_params.add_rands */
    float rand_scale_factor;    /* rand_params.rand_scale_factor */
    int32_t rand_seed;          /* rand_params.rand_seed */
    int32_t correct_com;        /* core.correct_com: shift all nodes by minus the mean of the
                                   cells' centres of mass after every step, src/GPUbounce.cu:1430-1440 */
    /* Variable stiffness (stiffnessParams.useDifferentStiffnesses): the initial softer cells
     * come from cs3d_initial_stiffness (src/GPUbounce.cu:616-692); from step phase_count on a
     * cell whose bond stiffness is not stiffness1 has pressure 0 and does not grow
     * (src/PressureKernels.cu:4-40); with soften_after_growth, more cells get stiffness2 at the
     * end of step div_time_steps + 2 (src/GPUbounce.cu:1340-1429): number_of_softer_cells of
     * them (roundf(fraction * cells) when fraction > 0), either distinct RANMAR picks
     * round(u * cells) from the division stream (choose_random_cell_indices) or the cells in
     * index order whose centre lies within (1 - closeness_to_center) of the largest distance
     * from the system's centre. */
    int32_t use_different_stiffnesses;
    float stiffness2;               /* stiffnessParams.softStiffFactor * Youngs_mod, src/GPUbounce.cu:2048 */
    int32_t phase_count;            /* core.phase_count */
    int32_t soften_after_growth;    /* !stiffnessParams.duringGrowth */
    int32_t number_of_softer_cells; /* stiffnessParams.numberOfSofterCells */
    float fraction_of_softer_cells; /* stiffnessParams.fractionOfSofterCells */
    int32_t choose_random_cell_indices; /* stiffnessParams.chooseRandomCellIndices */
    float closeness_to_center;      /* stiffnessParams.closenessToCenter */
    /* Mitotic index of internal cells (counting.count_only_internal_cells?): > 0 enables the
     * reference's num_cells_far test with this radius_cutoff, src/GPUbounce.cu:1288-1290,
     * :2538-2565; its results are read with cs3d_get_far_counts. */
    float count_internal_radius;
} cs3d_params;

/* ---- static mesh data ------------------------------------------------- */
typedef struct cs3d_topology {
    int32_t nn[3 * CS3D_SLOTS];     /* 0-based neighbours, [k*192 + node] */
    int32_t sign[CS3D_NODES];       /* orientation sign per node */
    float r0[3 * CS3D_SLOTS];       /* equilibrium bond lengths, [k*192 + node] */
    float theta0[3 * CS3D_SLOTS];   /* [node*3 + {aij, ajk, aik}] */
    int32_t faces[CS3D_FACES * 7];  /* C180_56 layout */
} cs3d_topology;

typedef struct cs3d_mesh {
    float xyz[CS3D_NODES * 3];      /* C180 file, row-major */
    int32_t nn[3 * CS3D_SLOTS];
    int32_t sign[CS3D_NODES];
    int32_t bonds[270 * 2];         /* C180C, 0-based */
    int32_t faces[CS3D_FACES * 7];
} cs3d_mesh;

/* RANMAR generator state, src/marsaglia.h:50-52 */
typedef struct cs3d_rng {
    float u[98];
    float c, cd, cm;
    int32_t i97, j97;
    int32_t ok;
} cs3d_rng;

/* Full inp.json contents, src/GPUbounce.cu:1914-2247 (all eight sections). */
typedef struct cs3d_config {
    /* core */
    int32_t max_cells;              /* MaxNoofC180s */
    float particle_mass, repulsion_range, attraction_range;
    float repulsion_strength, attraction_strength, youngs_mod, stiff_factor1;
    float viscotic_damping, internal_damping, gamma_visc, division_vol;
    int32_t random_z_offset; float z_offset;
    int32_t div_time_steps; float time_interval; int32_t restart;
    int32_t traj_write_int; int32_t non_div_time_steps;
    char traj_file_name[256]; int32_t binary_output;
    float max_pressure, min_pressure, growth_rate;
    int32_t check_sphericity, constrain_angles, do_adaptive_dt;
    float dt_max, dt_tol; int32_t phase_count; int32_t write_cont_force;
    char forces_file[256]; int32_t correct_com;
    /* counting */
    char mit_index_file[256]; int32_t count_only_internal; float radius_cutoff;
    int32_t overwrite_mit_ind; int32_t cell_count_int;
    /* population */
    int32_t do_pop_model; float total_food, regular_consumption, division_consumption;
    float death_release_food; int32_t cell_life_time; float max_pop;
    /* walls */
    int32_t use_walls; char perp_axis[8]; float d_axis, wall_len, wall_width, thresh_dist;
    /* divParams */
    int32_t use_div_plane_basis; float div_plane_basis[3];
    /* stiffnessParams */
    int32_t use_different_stiffnesses; float soft_stiff_factor; int32_t number_of_softer_cells;
    float fraction_of_softer_cells; int32_t during_growth, daught_same_stiffness;
    float closeness_to_center; int32_t start_at_pop, choose_random_cell_indices, recalc_r0;
    /* boxParams */
    int32_t use_rigid_box, use_pbcs; float box_length; float box_len[3];
    int32_t flatbox, rand_pos;
    /* rand_params */
    int32_t add_rands, rand_seed, rand_dist; float rand_scale_factor;
} cs3d_config;

typedef struct cs3d_ctx cs3d_ctx;

/* ---- host utilities (no GPU needed) ----------------------------------- */

/* Library version (major*10000 + minor*100 + patch).  No counterpart in the
 * reference. */
int cs3d_version(void);

/* Message for a status code.  No counterpart in the reference, which prints
 * its message and exits. */
const char *cs3d_strerror(int status);

/* Parse inp.json (// and C comments allowed) and apply the reference's
 * validation.  Replaces read_json_params, src/GPUbounce.cu:1914-2247. */
int cs3d_config_read_json(const char *path, cs3d_config *out, char *errbuf, int errlen);

/* Hot-path parameters from a parsed config: the conversions the reference
 * makes after reading the file (stiffness1 = stiffFactor1 x Youngs_mod,
 * src/GPUbounce.cu:1953; stiffness2 = softStiffFactor x Youngs_mod, :2048;
 * RANMAR seeds from rand_seed, :1796-1799, see cs3d_seed_map).  Returns
 * CS3D_E_UNSUPPORTED for features outside this library (population model,
 * walls, periodic box, adaptive time step, division-plane basis, recalc_r0). */
int cs3d_config_to_params(const cs3d_config *cfg, cs3d_params *out);

/* Read C180, C180NN, C180C, C180_pentahexa from a directory.  Replaces the
 * file readers of initialize_C180s and read_fullerene_nn,
 * src/GPUbounce.cu:1616-1627 and :1814-1888. */
int cs3d_mesh_read(const char *dir, cs3d_mesh *out);

/* Equilibrium bond lengths and angles from cell 0's initial positions
 * (192-stride arrays), host float arithmetic as src/GPUbounce.cu:1890-1908
 * (R0) and :909-938 (theta0). */
int cs3d_topology_build(const cs3d_mesh *mesh, const float *x0, const float *y0,
                        const float *z0, cs3d_topology *out);

/* RANMAR seeding, src/marsaglia.h:54-113.  Returns CS3D_E_ARG outside the
 * legal seed range (the reference exits). */
int cs3d_rng_init(cs3d_rng *rng, int ij, int kl);
/* RANMAR draws, src/marsaglia.h:115-144. */
int cs3d_rng_draw(cs3d_rng *rng, float *out, int len);
/* Marsaglia sphere point, src/RandomVector.h:8-24. */
int cs3d_rng_random_vector(cs3d_rng *rng, float n[3]);
/* rand_seed -> (ij, kl): (seed, 100*seed) as src/GPUbounce.cu:1796-1799 for
 * 0 <= seed <= 300; larger seeds fold into the legal range
 * (seed mod 31329, 100*seed mod 30082). */
int cs3d_seed_map(int seed, int *ij, int *kl);

/* Bond stiffness (Young's modulus) of the n_cells initial cells, src/GPUbounce.cu:616-692:
 * stiffness1 for every cell; with useDifferentStiffnesses stiffness2 for the cells whose centre
 * of mass lies within closenessToCenter of the largest distance from the system's centre (when
 * 0 < closenessToCenter < 1), else for numberOfSofterCells cells (roundf(fraction * n) when
 * 0 < fraction < 1): the first ones in a rigid box, RANMAR picks round(u * n) from rng
 * otherwise.  X/Y/Z are 192-stride.  Returns CS3D_E_CONFIG when more softer cells than cells
 * are requested (the reference exits with 12516). */
int cs3d_initial_stiffness(const cs3d_config *cfg, int n_cells, const float *X, const float *Y,
                           const float *Z, cs3d_rng *rng, float *youngs);

/* Initial cell placement, src/GPUbounce.cu:1598-1774 (lattice or random
 * insertion with RANMAR draws).  X/Y/Z have capacity n_cells*192. */
int cs3d_init_positions(const cs3d_config *cfg, const cs3d_mesh *mesh, int n_cells,
                        cs3d_rng *rng, float *X, float *Y, float *Z);

/* Binary trajectory writer, src/GPUbounce.cu:1007-1018 (header),
 * :2446-2477 (frames), :1508-1511 (final cell count).  Read by
 * scripts/celldiv.py. */
typedef struct cs3d_traj cs3d_traj;
int cs3d_traj_open(const char *path, int max_cells, int variable_stiffness, int max_frames,
                   cs3d_traj **out);
int cs3d_traj_write_frame(cs3d_traj *t, int step, int frame, int n_cells, const float *X,
                          const float *Y, const float *Z, const int32_t *types);
int cs3d_traj_close(cs3d_traj *t, int final_cells);

/* ---- device context --------------------------------------------------- */

/* One simulation with room for capacity_cells cells.  stream may be NULL
 * (the context creates its own).  Replaces the allocation block of main,
 * src/GPUbounce.cu:358-527. */
int cs3d_create(const cs3d_params *params, const cs3d_topology *topo, int capacity_cells,
                int device, void *stream, cs3d_ctx **out);

/* A batch of n_inst independent simulations stepped together (per-instance
 * parameters, seeds, boxes and capacities).  No counterpart in the
 * reference, which runs one simulation per process. */
int cs3d_create_ensemble(int n_inst, const cs3d_params *params, const cs3d_topology *topo,
                         const int *capacity_cells, int device, void *stream, cs3d_ctx **out);

/* Load the state of instance inst: n_cells cells, 192-stride SoA.
 * V*, pressure and youngs may be NULL (zeros, min_pressure, stiffness1 --
 * the reference's defaults, src/GPUbounce.cu:449-451, :867-871, :617-620).
 * The initial centre of mass, grid and first force evaluation
 * (src/GPUbounce.cu:739-763, :978-1004) run before the next step or read. */
int cs3d_load_state(cs3d_ctx *ctx, int inst, int n_cells, const float *X, const float *Y,
                    const float *Z, const float *VX, const float *VY, const float *VZ,
                    const float *pressure, const float *youngs);

/* Replace the RANMAR state of instance inst (e.g. after host-side draws
 * for random placement).  The reference keeps one RANMAR state per process
 * in file-scope variables (src/marsaglia.h:50-51); an ensemble has one per
 * instance, so it is set and read through these two calls. */
int cs3d_set_rng(cs3d_ctx *ctx, int inst, const cs3d_rng *rng);
/* Current RANMAR state of instance inst (the stream the divisions draw from). */
int cs3d_get_rng(cs3d_ctx *ctx, int inst, cs3d_rng *rng);

/* Neighbour-list skin by population range, for every instance: an instance
 * with at least min_cells[k] cells (ascending bounds) steps with skins[k],
 * below min_cells[0] with the context's skin (CS3D_OPT_SKIN).  The device
 * applies it at the start of each step from the instance's current cell
 * count; a change takes effect with a whole-instance list rebuild in that
 * step.  The skin changes no result -- the contact-pair sets and the order
 * in which the force sums run do not depend on it -- only the time (longer
 * lists against fewer rebuilds), so a schedule picked by timing
 * (cellsim3d_b200.autotune) is safe to apply.  n = 0 clears it.  No
 * counterpart in the reference, whose contact grid has a fixed spacing
 * (src/GPUbounce.cu:756) and whose launch shapes are fixed (one block per
 * cell, src/GPUbounce.cu:1059-1151).  CS3D_E_ARG for n < 0, n >
 * CS3D_SKIN_RANGES, bounds not strictly ascending or below 1, or a skin
 * outside (0.002, 1]. */
#define CS3D_SKIN_RANGES 8
int cs3d_set_skin_schedule(cs3d_ctx *ctx, int n, const int *min_cells, const float *skins);

/* Advance every instance by n_steps timesteps of src/GPUbounce.cu:1055-1338.
 * Returns CS3D_E_DEVICE_FLAGS or CS3D_E_CAPACITY if a kernel raised an
 * error bit (see cs3d_last_error). */
int cs3d_step(cs3d_ctx *ctx, int n_steps);

/* Read back instance inst.  Any output pointer may be NULL.  Replaces the
 * device-to-host copies before a trajectory frame and the force file,
 * src/GPUbounce.cu:1447-1449 and :1458-1471. */
int cs3d_get_state(cs3d_ctx *ctx, int inst, int *n_cells, float *X, float *Y, float *Z,
                   float *VX, float *VY, float *VZ, float *pressure, float *youngs);

/* Start reading instance inst back without waiting for it, so that the next
 * cs3d_step overlaps the device-to-host copy (the reference reads each frame
 * back on its step loop's thread and the GPU idles meanwhile,
 * src/GPUbounce.cu:1443-1475, WriteBinaryTraj :2446-2477).  The cell count is
 * read first (a short synchronous read) and stored in *n_cells; the arrays
 * are then gathered on the context's stream into one of two device staging
 * slots (slot 0 or 1) and copied to the caller's buffers on a separate copy
 * stream, one cudaMemcpyAsync per array.  Output pointers may be NULL; they
 * should be page-locked (cs3d_host_alloc) for the copy to be asynchronous.
 * The buffers must stay valid and unread until cs3d_wait_state(ctx, slot)
 * returns.  A later call on the same slot first waits (on the device) for
 * that slot's previous copy.  No counterpart in the reference. */
int cs3d_get_state_async(cs3d_ctx *ctx, int inst, int slot, int *n_cells, float *X, float *Y, float *Z,
                         float *VX, float *VY, float *VZ, float *pressure, float *youngs);

/* Wait until the copies started by cs3d_get_state_async on `slot` have
 * landed in the caller's buffers.  Returns CS3D_OK at once if none is
 * pending.  No counterpart in the reference. */
int cs3d_wait_state(cs3d_ctx *ctx, int slot);

/* Page-locked host memory for cs3d_get_state_async and cs3d_load_state
 * (cudaHostAlloc / cudaFreeHost), for callers that do not link the CUDA
 * runtime themselves.  No counterpart in the reference. */
int cs3d_host_alloc(size_t bytes, void **ptr);
int cs3d_host_free(void *ptr);

/* Conservative (fConList) and dissipative (fDisList) forces of the last
 * evaluation, 192-stride SoA.  The conservative force is what the force
 * file (write_cont_force, src/GPUbounce.cu:1456-1473) reads back. */
int cs3d_get_forces(cs3d_ctx *ctx, int inst, float *FCX, float *FCY, float *FCZ,
                    float *FDX, float *FDY, float *FDZ);

/* Histogram of the volumes of instance inst's cells at the current positions (centre of mass
 * and volume of src/volume.cu:5-163 in FP64, computed on the device; the analysis that the
 * reference's scripts do offline): counts[0] below lo, counts[1..nbins] the equal bins of
 * [lo, hi), counts[nbins + 1] at or above hi.  volumes (may be NULL) receives every cell's
 * volume. */
int cs3d_volume_histogram(cs3d_ctx *ctx, int inst, float lo, float hi, int nbins, int64_t *counts,
                          float *volumes);

/* Division steps at which cells were discounted from the mitotic index as far from the
 * system's centre (count_internal_radius > 0; src/GPUbounce.cu:1288-1290, :2538-2565):
 * pairs (step, count) into out[2 * max_entries]; *n_entries = the number recorded. */
int cs3d_get_far_counts(cs3d_ctx *ctx, int inst, int32_t *out, int max_entries, int *n_entries);

/* Langevin random force of the last step (zeros when add_rands is off or
 * before the first step), 192-stride SoA.  No counterpart in the reference
 * (its fRanList stays on the device). */
int cs3d_get_random_force(cs3d_ctx *ctx, int inst, float *FRX, float *FRY, float *FRZ);

/* Per-cell centre of mass (3*n), volume, area and bounding box (6*n:
 * minx maxx miny maxy minz maxz) as of the last step.  The reference reads
 * back only the volumes (src/GPUbounce.cu:1471); the rest stays on its
 * device (CenterOfMass, src/centermass.cu:8-50; bounding_boxes,
 * src/propagatebound.cu:10-205). */
int cs3d_get_cells(cs3d_ctx *ctx, int inst, float *cm, float *volume, float *area,
                   float *aabb);

/* The neighbour-grid extents (Minx[0..5]) and divisions used by the next
 * force evaluation (the reference's minmaxpre/minmaxpost and grid set-up,
 * src/propagatebound.cu:10-205, whose results stay on the device). */
int cs3d_get_grid(cs3d_ctx *ctx, int inst, float minmax[6], int divs[3]);

/* Options of this library's neighbour lists and pair recording.  No
 * counterpart in the reference. */
#define CS3D_OPT_RECORD_PAIRS  1   /* value 0/1: record the contact pairs used */
#define CS3D_OPT_SKIN          2   /* value = skin length in units of 1e-6 */
#define CS3D_OPT_PAIR_CAPACITY 3   /* value = max recorded pairs */
#define CS3D_OPT_REBUILD       4   /* value ignored: rebuild every neighbour list at the next step */
#define CS3D_OPT_HALO_STATS    5   /* value 0/1: count the distinct contact-candidate nodes of each cell
                                      at every list build (cs3d_get_stats [5]); off by default, as the
                                      count costs the build a shared-memory atomic per entry */
int cs3d_set_option(cs3d_ctx *ctx, int option, long long value);

/* Contact pairs recorded during the last force evaluation (requires
 * CS3D_OPT_RECORD_PAIRS).  kind 0: conservative (strict cut-off,
 * src/propagate.cu:421); kind 1: dissipative (src/propagate.cu:641).
 * out receives (cell_a, node_i, cell_b, node_j) quadruples. */
int cs3d_get_pairs(cs3d_ctx *ctx, int inst, int kind, int32_t *out, long long max_pairs,
                   long long *count);

/* Division events (step, parent, daughter) since creation: the cells that
 * cell_division (src/postscriptinit.cu:148-256) splits each step.  The
 * reference does not record them. */
int cs3d_get_events(cs3d_ctx *ctx, int inst, int32_t *out, int max_events, int *count);

/* Error bits raised on the device for instance inst (OR of CS3D_ERRBIT_*).
 * Where the reference traps or exits (the bits' comments cite where), this
 * library sets a bit and the step returns an error status. */
int cs3d_last_error(cs3d_ctx *ctx, int inst, uint32_t *bits);

/* Counters of this library's neighbour lists (no counterpart in the
 * reference): [0] steps, [1] neighbour-list rebuilds, [2] max entries per node
 * seen, [3] max candidate cells per cell seen, [4] kernel launches per step,
 * [5] max distinct contact-candidate nodes (of other cells) per cell seen
 * (counted only with CS3D_OPT_HALO_STATS, else 0),
 * [6] cell neighbour lists built (cumulative), [7] of the rebuilds [1], those
 * that only the rule for dividing instances called for (a division in the
 * step and a node more than a quarter of the skin from its anchor, with no
 * node past half the skin). */
int cs3d_get_stats(cs3d_ctx *ctx, long long *stats, int n);

/* Profiling pass: n_steps steps launched kernel by kernel (not as a graph)
 * with a CUDA event after each launch on the context's stream; kernel_ms
 * receives the average time of each launch slot of a step, names a
 * comma-separated list of their names.  Slots are matched by launch order,
 * so the steps of one call should launch the same kernels: a call that
 * spans the last division step or a softening step mixes kernels within a
 * slot.  No counterpart in the reference. */
int cs3d_profile_step(cs3d_ctx *ctx, int n_steps, float *kernel_ms, char *names, int names_len,
                      int max_kernels, int *n_kernels);

/* ---- force evaluation without allocation ------------------------------ */

/* Largest system cs3d_forces_static accepts. */
#define CS3D_STATIC_MAX_CELLS 64

/* Forces of one system of n_cells <= CS3D_STATIC_MAX_CELLS cells -- the
 * force evaluation that cs3d_load_state triggers, with the same kernels and
 * the same results -- computed without allocating any memory.
 *
 * No counterpart in the reference.  It is meant for callers that cannot
 * allocate GPU memory: code running inside a host that has already
 * partitioned the device (a memory pool or arena owned by someone else), a
 * real-time loop that must never call cudaMalloc/cudaFree (they synchronise
 * the device), or a plugin host that forbids allocation in callbacks.  The
 * caller passes device pointers to inputs and outputs it owns; everything
 * else the kernels need (the contact lists, grids and per-cell data) lives
 * in one file-scope static device array of this library (4.2 MB, held
 * by every GPU that loads the library until the process exits).
 *
 * Inputs (device, 192-stride SoA as cs3d_load_state): X, Y, Z, VX, VY, VZ
 * (VX/VY/VZ may be NULL: zero velocity), pressure and youngs (device, per
 * cell; NULL: min_pressure and stiffness1).  Outputs (device, 192-stride):
 * the conservative and dissipative forces; slots 180..191 are set to zero.
 * stream may be NULL (legacy default stream).
 *
 * The first call on a device resolves the static array's device address
 * (cudaGetSymbolAddress) and sets kernel attributes; make that first call
 * before any stream capture.  The address is kept for the life of the
 * process: after a cudaDeviceReset of that device the entry point must not
 * be called again.  Every call shares the one static array, so calls that
 * overlap on the GPU (different streams or host threads) race: serialise
 * them.  Every call copies the error word back to the host and synchronises
 * its stream before returning.  With correct_com set, the positions are
 * shifted by the centre-of-mass correction before the forces are evaluated,
 * as in cs3d_load_state.  Returns CS3D_E_ARG for n_cells outside
 * [1, CS3D_STATIC_MAX_CELLS] or a NULL required pointer. */
int cs3d_forces_static(const cs3d_params *params, const cs3d_topology *topo, int n_cells,
                       const float *X, const float *Y, const float *Z,
                       const float *VX, const float *VY, const float *VZ,
                       const float *pressure, const float *youngs,
                       float *FCX, float *FCY, float *FCZ, float *FDX, float *FDY, float *FDZ,
                       void *stream);

/* Device time of the last cs3d_step call (ms, CUDA events).  No counterpart
 * in the reference. */
int cs3d_last_step_ms(cs3d_ctx *ctx, float *ms);

/* Release the context and its device memory.  Replaces the cudaFree block at
 * the end of main, src/GPUbounce.cu:1549-1566. */
int cs3d_destroy(cs3d_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* CS3D_H */
