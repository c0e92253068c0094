// cs3d_host.cpp -- host-side utilities of libcs3d.so (no GPU needed):
// inp.json parsing, mesh files, static bond/angle data, RANMAR, initial
// placement and the binary trajectory writer.  Float arithmetic here follows
// the reference's host code expression by expression; the library is built
// with -ffp-contract=off so no FMA contraction changes a rounding.
#include "../../include/cs3d.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Minimal JSON reader accepting // and /* */ comments, like jsoncpp 0.7.0's
// Reader with comments allowed (the reference's inp.json relies on this).
// ---------------------------------------------------------------------------
struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0;
    bool is_int = false;
    std::string str;
    std::vector<JVal> arr;
    std::map<std::string, JVal> obj;
};

struct JParser {
    const char *p, *end;
    std::string err;
    int line = 1;

    void skip_ws() {
        while (p < end) {
            if (*p == '\n') { ++line; ++p; }
            else if (*p == ' ' || *p == '\t' || *p == '\r') ++p;
            else if (*p == '/' && p + 1 < end && p[1] == '/') {
                while (p < end && *p != '\n') ++p;
            } else if (*p == '/' && p + 1 < end && p[1] == '*') {
                p += 2;
                while (p + 1 < end && !(p[0] == '*' && p[1] == '/')) { if (*p == '\n') ++line; ++p; }
                if (p + 1 >= end) { err = "unterminated comment"; p = end; return; }
                p += 2;
            } else break;
        }
    }
    bool fail(const char *m) {
        if (err.empty()) err = std::string(m) + " at line " + std::to_string(line);
        return false;
    }
    bool parse_string(std::string &out) {
        if (p >= end || *p != '"') return fail("expected string");
        ++p;
        while (p < end && *p != '"') {
            if (*p == '\\' && p + 1 < end) {
                ++p;
                char c = *p++;
                switch (c) {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'u': out += '?'; p += (end - p >= 4 ? 4 : end - p); break;
                default: out += c;
                }
            } else {
                if (*p == '\n') ++line;
                out += *p++;
            }
        }
        if (p >= end) return fail("unterminated string");
        ++p;
        return true;
    }
    bool parse(JVal &v) {
        skip_ws();
        if (!err.empty()) return false;
        if (p >= end) return fail("unexpected end");
        char c = *p;
        if (c == '{') {
            v.kind = JVal::Obj;
            ++p;
            skip_ws();
            if (p < end && *p == '}') { ++p; return true; }
            while (true) {
                skip_ws();
                std::string key;
                if (!parse_string(key)) return false;
                skip_ws();
                if (p >= end || *p != ':') return fail("expected ':'");
                ++p;
                JVal child;
                if (!parse(child)) return false;
                v.obj[key] = std::move(child);
                skip_ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == '}') { ++p; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = JVal::Arr;
            ++p;
            skip_ws();
            if (p < end && *p == ']') { ++p; return true; }
            while (true) {
                JVal child;
                if (!parse(child)) return false;
                v.arr.push_back(std::move(child));
                skip_ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == ']') { ++p; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') { v.kind = JVal::Str; return parse_string(v.str); }
        if (!strncmp(p, "true", 4)) { v.kind = JVal::Bool; v.b = true; p += 4; return true; }
        if (!strncmp(p, "false", 5)) { v.kind = JVal::Bool; v.b = false; p += 5; return true; }
        if (!strncmp(p, "null", 4)) { v.kind = JVal::Null; p += 4; return true; }
        if (c == '-' || (c >= '0' && c <= '9')) {
            const char *s = p;
            bool isint = true;
            if (*p == '-') ++p;
            while (p < end && ((*p >= '0' && *p <= '9') || *p == '.' || *p == 'e' || *p == 'E' ||
                               *p == '+' || *p == '-')) {
                if (*p == '.' || *p == 'e' || *p == 'E') isint = false;
                ++p;
            }
            std::string tok(s, p);
            char *ep = nullptr;
            v.kind = JVal::Num;
            v.num = strtod(tok.c_str(), &ep);
            v.is_int = isint;
            if (!ep || *ep) return fail("bad number");
            return true;
        }
        return fail("unexpected character");
    }
};

// jsoncpp conversions: a missing member reads as null -> 0 / false / "".
const JVal *member(const JVal &o, const char *k) {
    if (o.kind != JVal::Obj) return nullptr;
    auto it = o.obj.find(k);
    return it == o.obj.end() ? nullptr : &it->second;
}
int as_int(const JVal &o, const char *k) {
    const JVal *v = member(o, k);
    if (!v) return 0;
    if (v->kind == JVal::Num) return (int)v->num;
    if (v->kind == JVal::Bool) return v->b ? 1 : 0;
    return 0;
}
float as_float(const JVal &o, const char *k) {
    const JVal *v = member(o, k);
    if (!v) return 0.0f;
    if (v->kind == JVal::Num) return (float)v->num;
    if (v->kind == JVal::Bool) return v->b ? 1.0f : 0.0f;
    return 0.0f;
}
int as_bool(const JVal &o, const char *k) {
    const JVal *v = member(o, k);
    if (!v) return 0;
    if (v->kind == JVal::Num) return v->num != 0.0;
    if (v->kind == JVal::Bool) return v->b;
    return 0;
}
void as_string(const JVal &o, const char *k, char *dst, size_t n) {
    const JVal *v = member(o, k);
    std::string s = (v && v->kind == JVal::Str) ? v->str : std::string();
    snprintf(dst, n, "%s", s.c_str());
}

void set_err(char *errbuf, int errlen, const std::string &m) {
    if (errbuf && errlen > 0) snprintf(errbuf, (size_t)errlen, "%s", m.c_str());
}

float f3mag(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

}  // namespace

extern "C" {

int cs3d_version(void) { return 10000; }

const char *cs3d_strerror(int s)
{
    switch (s) {
    case CS3D_OK: return "ok";
    case CS3D_E_ARG: return "invalid argument";
    case CS3D_E_CUDA: return "CUDA runtime error";
    case CS3D_E_NOMEM: return "out of memory";
    case CS3D_E_IO: return "file could not be opened or read";
    case CS3D_E_PARSE: return "inp.json could not be parsed";
    case CS3D_E_CONFIG: return "invalid parameter value";
    case CS3D_E_DEVICE_FLAGS: return "a kernel raised an error bit";
    case CS3D_E_CAPACITY: return "population exceeded the allocated capacity";
    case CS3D_E_UNSUPPORTED: return "feature not supported by this library";
    default: return "unknown status";
    }
}

// read_json_params, src/GPUbounce.cu:1914-2247 (sections, keys, defaults and
// the validation block :2076-2244).
int cs3d_config_read_json(const char *path, cs3d_config *out, char *errbuf, int errlen)
{
    if (!path || !out) return CS3D_E_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) { set_err(errbuf, errlen, std::string("cannot open ") + path); return CS3D_E_IO; }
    std::string text;
    char buf[65536];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, k);
    fclose(f);
    JParser jp{text.data(), text.data() + text.size()};
    JVal root;
    if (!jp.parse(root)) { set_err(errbuf, errlen, "Failed to parse " + std::string(path) + ": " + jp.err); return CS3D_E_PARSE; }
    if (root.kind != JVal::Obj) { set_err(errbuf, errlen, "top level is not an object"); return CS3D_E_PARSE; }
    memset(out, 0, sizeof *out);
    const JVal *core = member(root, "core");
    if (!core || core->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load core simulation parameters"); return CS3D_E_PARSE; }
    const JVal &c = *core;
    out->max_cells = as_int(c, "MaxNoofC180s");
    out->particle_mass = as_float(c, "particle_mass");
    out->repulsion_range = as_float(c, "repulsion_range");
    out->attraction_range = as_float(c, "attraction_range");
    out->repulsion_strength = as_float(c, "repulsion_strength");
    out->attraction_strength = as_float(c, "attraction_strength");
    out->youngs_mod = as_float(c, "Youngs_mod");
    out->stiff_factor1 = as_float(c, "stiffFactor1");
    out->viscotic_damping = as_float(c, "viscotic_damping");
    out->internal_damping = as_float(c, "internal_damping");
    out->division_vol = as_float(c, "division_Vol");
    out->random_z_offset = as_int(c, "random_z_offset?");
    out->z_offset = as_float(c, "z_offset");
    out->div_time_steps = (int)as_float(c, "div_time_steps");
    out->time_interval = as_float(c, "time_interval");
    out->restart = as_int(c, "Restart");
    out->traj_write_int = as_int(c, "trajWriteInt");
    out->non_div_time_steps = as_int(c, "non_div_time_steps");
    as_string(c, "trajFileName", out->traj_file_name, sizeof out->traj_file_name);
    out->binary_output = as_bool(c, "binaryOutput");
    out->max_pressure = as_float(c, "maxPressure");
    out->min_pressure = as_float(c, "minPressure");
    out->gamma_visc = as_float(c, "gamma_visc");
    out->growth_rate = as_float(c, "growth_rate");
    out->check_sphericity = as_bool(c, "checkSphericity");
    out->constrain_angles = as_bool(c, "constrainAngles");
    out->dt_max = as_float(c, "dt_max");
    out->dt_tol = as_float(c, "dt_tol");
    out->do_adaptive_dt = as_bool(c, "doAdaptive_dt");
    out->phase_count = as_int(c, "phase_count");
    out->write_cont_force = as_bool(c, "write_cont_force");
    as_string(c, "forces_file", out->forces_file, sizeof out->forces_file);
    out->correct_com = as_bool(c, "correct_com");

    const JVal *cnt = member(root, "counting");
    if (!cnt || cnt->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load counting parameters"); return CS3D_E_PARSE; }
    as_string(*cnt, "mit-index_file_name", out->mit_index_file, sizeof out->mit_index_file);
    out->count_only_internal = as_bool(*cnt, "count_only_internal_cells?");
    out->radius_cutoff = as_float(*cnt, "radius_cutoff");
    out->overwrite_mit_ind = as_bool(*cnt, "overwrite_mit_ind_file?");
    out->cell_count_int = as_int(*cnt, "cell_count_int");

    const JVal *pop = member(root, "population");
    if (!pop || pop->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load population parameters"); return CS3D_E_PARSE; }
    out->do_pop_model = as_int(*pop, "doPopModel");
    out->total_food = as_float(*pop, "totalFood");
    out->regular_consumption = as_float(*pop, "regular_consumption");
    out->division_consumption = as_float(*pop, "division_consumption");
    out->death_release_food = as_float(*pop, "death_release_food");
    out->cell_life_time = as_int(*pop, "cellLifeTime");
    out->max_pop = as_float(*pop, "max_pop");

    const JVal *w = member(root, "walls");
    if (!w || w->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load wall parameters"); return CS3D_E_PARSE; }
    out->use_walls = as_int(*w, "useWalls");
    as_string(*w, "perpAxis", out->perp_axis, sizeof out->perp_axis);
    out->d_axis = as_float(*w, "dAxis");
    out->wall_len = as_float(*w, "wallLen");
    out->wall_width = as_float(*w, "wallWidth");
    out->thresh_dist = as_float(*w, "threshDist");

    const JVal *dp = member(root, "divParams");
    if (!dp || dp->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load division parameters"); return CS3D_E_PARSE; }
    out->use_div_plane_basis = as_int(*dp, "useDivPlaneBasis");
    out->div_plane_basis[0] = as_float(*dp, "divPlaneBasisX");
    out->div_plane_basis[1] = as_float(*dp, "divPlaneBasisY");
    out->div_plane_basis[2] = as_float(*dp, "divPlaneBasisZ");

    const JVal *sp = member(root, "stiffnessParams");
    if (!sp || sp->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load stiffness parameters"); return CS3D_E_PARSE; }
    out->use_different_stiffnesses = as_bool(*sp, "useDifferentStiffnesses");
    out->soft_stiff_factor = as_float(*sp, "softStiffFactor");
    out->number_of_softer_cells = as_int(*sp, "numberOfSofterCells");
    out->during_growth = as_bool(*sp, "duringGrowth");
    out->closeness_to_center = as_float(*sp, "closenessToCenter");
    out->start_at_pop = as_int(*sp, "startAtPop");
    out->fraction_of_softer_cells = as_float(*sp, "fractionOfSofterCells");
    out->choose_random_cell_indices = as_bool(*sp, "chooseRandomCellIndices");
    out->daught_same_stiffness = as_bool(*sp, "daughtSameStiffness");
    out->recalc_r0 = as_bool(*sp, "recalc_r0");

    const JVal *bp = member(root, "boxParams");
    if (!bp || bp->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load box parameters"); return CS3D_E_PARSE; }
    out->use_rigid_box = as_bool(*bp, "useRigidSimulationBox");
    out->use_pbcs = as_bool(*bp, "usePBCs");
    out->box_length = as_float(*bp, "boxLength");
    out->box_len[0] = as_float(*bp, "box_len_x");
    out->box_len[1] = as_float(*bp, "box_len_y");
    out->box_len[2] = as_float(*bp, "box_len_z");
    out->flatbox = as_bool(*bp, "flatbox");
    out->rand_pos = as_bool(*bp, "rand_pos");

    if (out->random_z_offset == 0) out->z_offset = 0.0f;
    if (out->dt_tol > out->dt_max || out->dt_max <= 0 || out->dt_tol < 0) {
        set_err(errbuf, errlen, "Invalid time step parameters");
        return CS3D_E_CONFIG;
    }

    const JVal *rp = member(root, "rand_params");
    if (!rp || rp->kind == JVal::Null) { set_err(errbuf, errlen, "Cannot load randomness parameters"); return CS3D_E_PARSE; }
    out->add_rands = as_bool(*rp, "add_rands");
    out->rand_seed = as_int(*rp, "rand_seed");
    out->rand_dist = as_int(*rp, "rand_dist");
    out->rand_scale_factor = as_float(*rp, "rand_scale_factor");

    if (out->radius_cutoff < 0.4f || out->radius_cutoff > 0.8f || out->radius_cutoff < 0)
        out->count_only_internal = 0;
    if (out->traj_write_int == 0) out->traj_write_int = 1;
    if (out->cell_count_int == 0) out->cell_count_int = 1;
    if (out->traj_write_int > out->div_time_steps + out->non_div_time_steps) {
        set_err(errbuf, errlen, "Trajectory write interval is too large");
        return CS3D_E_CONFIG;
    }
    if (out->div_time_steps % out->traj_write_int != 0) {
        set_err(errbuf, errlen, "Invalid trajectory write interval. Time steps must be divisible by it.");
        return CS3D_E_CONFIG;
    }
    if (out->cell_count_int > out->div_time_steps) {
        set_err(errbuf, errlen, "New cell counting interval is too large.");
        return CS3D_E_CONFIG;
    }
    if (out->non_div_time_steps <= 0) out->non_div_time_steps = 0;
    if (out->do_pop_model != 1) out->do_pop_model = 0;
    if (out->max_pressure < 0) out->do_pop_model = 0;
    if (!(out->closeness_to_center >= 0 && out->closeness_to_center <= 1)) {
        set_err(errbuf, errlen, "closenessToCenter is not in [0, 1]");
        return CS3D_E_CONFIG;
    }
    if (out->use_walls && out->use_rigid_box) {
        set_err(errbuf, errlen, "Cannot use infinite XY walls and rigid simulation box simultaneously.");
        return CS3D_E_CONFIG;
    }
    if (out->fraction_of_softer_cells > 1.0f) {
        set_err(errbuf, errlen, "Softer cell fraction is > 1");
        return CS3D_E_CONFIG;
    }
    return CS3D_OK;
}

int cs3d_seed_map(int seed, int *ij, int *kl)
{
    if (!ij || !kl) return CS3D_E_ARG;
    long s = seed;
    if (s >= 0 && s <= 300) { *ij = (int)s; *kl = (int)(100 * s); return CS3D_OK; }
    if (s < 0) s = -s;
    *ij = (int)(s % 31329);
    *kl = (int)((100 * s) % 30082);
    return CS3D_OK;
}

int cs3d_config_to_params(const cs3d_config *c, cs3d_params *p)
{
    if (!c || !p) return CS3D_E_ARG;
    memset(p, 0, sizeof *p);
    p->particle_mass = c->particle_mass;
    p->repulsion_range = c->repulsion_range;
    p->attraction_range = c->attraction_range;
    p->repulsion_strength = c->repulsion_strength;
    p->attraction_strength = c->attraction_strength;
    p->youngs_mod = c->youngs_mod;
    p->stiffness1 = c->stiff_factor1 * c->youngs_mod;
    p->internal_damping = c->internal_damping;
    p->viscotic_damping = c->viscotic_damping;
    p->gamma_visc = c->gamma_visc;
    p->division_vol = c->division_vol;
    p->time_interval = c->time_interval;
    p->max_pressure = c->max_pressure;
    p->min_pressure = c->min_pressure;
    p->growth_rate = c->growth_rate;   // the population model (doPopModel) is refused below
    p->thresh_dist = c->thresh_dist;
    p->box_len[0] = c->box_len[0];
    p->box_len[1] = c->box_len[1];
    p->box_len[2] = c->box_len[2];
    p->check_sphericity = c->check_sphericity;
    p->constrain_angles = c->constrain_angles;
    p->use_rigid_box = c->use_rigid_box;
    p->daught_same_stiffness = c->daught_same_stiffness;
    p->div_time_steps = c->div_time_steps;
    cs3d_seed_map(c->rand_seed, &p->rng_ij, &p->rng_kl);
    p->add_rands = c->add_rands ? 1 : 0;
    p->rand_scale_factor = c->rand_scale_factor;
    p->rand_seed = c->rand_seed;   // <= 0: the caller picks one (the reference seeds from time())
    p->correct_com = c->correct_com ? 1 : 0;
    p->use_different_stiffnesses = c->use_different_stiffnesses ? 1 : 0;
    p->stiffness2 = c->soft_stiff_factor * c->youngs_mod;
    p->phase_count = c->phase_count;
    p->soften_after_growth = c->use_different_stiffnesses && !c->during_growth ? 1 : 0;
    p->number_of_softer_cells = c->number_of_softer_cells;
    p->fraction_of_softer_cells = c->fraction_of_softer_cells;
    p->choose_random_cell_indices = c->choose_random_cell_indices ? 1 : 0;
    p->closeness_to_center = c->closeness_to_center;
    p->count_internal_radius = c->count_only_internal ? c->radius_cutoff : 0.0f;
    // Features of the reference this library leaves out (all off in the
    // reference's shipped inp.json and in every benchmark configuration).
    // recalc_r0: the reference's CalculateR0 (src/BondKernels.cu:3-37) stores
    // per-cell mean bond lengths into the 3x192 per-bond table d_R0
    // (src/GPUbounce.cu:400), past its end from cell 576 on, so the behaviour
    // it asks for is not defined.
    if (c->do_pop_model || c->use_div_plane_basis || c->use_walls || c->use_pbcs || c->do_adaptive_dt ||
        (c->use_different_stiffnesses && c->recalc_r0))
        return CS3D_E_UNSUPPORTED;
    return CS3D_OK;
}

// Mesh readers: C180 via fscanf("%f") (src/GPUbounce.cu:1616-1627), C180NN
// "%d,%d,%d,%d" 1-based (:1822-1836), C180C "%d,%d" (:1840-1852),
// C180_pentahexa 12 pentagons + 80 hexagons, 0-based (:1858-1888).
int cs3d_mesh_read(const char *dir, cs3d_mesh *m)
{
    if (!dir || !m) return CS3D_E_ARG;
    memset(m, 0, sizeof *m);
    std::string d(dir);
    if (!d.empty() && d.back() != '/') d += '/';
    FILE *f = fopen((d + "C180").c_str(), "r");
    if (!f) return CS3D_E_IO;
    for (int a = 0; a < 180; ++a)
        if (fscanf(f, "%f %f %f", &m->xyz[3 * a], &m->xyz[3 * a + 1], &m->xyz[3 * a + 2]) != 3) { fclose(f); return CS3D_E_IO; }
    fclose(f);
    f = fopen((d + "C180NN").c_str(), "r");
    if (!f) return CS3D_E_IO;
    for (int i = 0; i < 180; ++i) {
        int n1, n2, n3, s;
        if (fscanf(f, "%d,%d,%d,%d", &n1, &n2, &n3, &s) != 4) { fclose(f); return CS3D_E_IO; }
        m->nn[i] = n1 - 1;
        m->nn[192 + i] = n2 - 1;
        m->nn[384 + i] = n3 - 1;
        m->sign[i] = s;
    }
    fclose(f);
    f = fopen((d + "C180C").c_str(), "r");
    if (!f) return CS3D_E_IO;
    for (int i = 0; i < 270; ++i) {
        int a, b;
        if (fscanf(f, "%d,%d", &a, &b) != 2) { fclose(f); return CS3D_E_IO; }
        m->bonds[2 * i] = a - 1;
        m->bonds[2 * i + 1] = b - 1;
    }
    fclose(f);
    f = fopen((d + "C180_pentahexa").c_str(), "r");
    if (!f) return CS3D_E_IO;
    for (int i = 0; i < 12; ++i) {
        int v[5];
        if (fscanf(f, "%d %d %d %d %d", &v[0], &v[1], &v[2], &v[3], &v[4]) != 5) { fclose(f); return CS3D_E_IO; }
        for (int q = 0; q < 5; ++q) m->faces[i * 7 + q] = v[q];
        m->faces[i * 7 + 5] = v[0];
        m->faces[i * 7 + 6] = v[0];
    }
    for (int i = 0; i < 80; ++i) {
        int v[6];
        if (fscanf(f, "%d %d %d %d %d %d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]) != 6) { fclose(f); return CS3D_E_IO; }
        for (int q = 0; q < 6; ++q) m->faces[84 + i * 7 + q] = v[q];
        m->faces[84 + i * 7 + 6] = v[0];
    }
    fclose(f);
    return CS3D_OK;
}

// R0: src/GPUbounce.cu:1890-1908; theta0: :909-938.  Float host arithmetic.
int cs3d_topology_build(const cs3d_mesh *m, const float *X, const float *Y, const float *Z,
                        cs3d_topology *t)
{
    if (!m || !X || !Y || !Z || !t) return CS3D_E_ARG;
    memset(t, 0, sizeof *t);
    memcpy(t->nn, m->nn, sizeof t->nn);
    memcpy(t->sign, m->sign, sizeof t->sign);
    memcpy(t->faces, m->faces, sizeof t->faces);
    for (int i = 0; i < 180; ++i)
        for (int k = 0; k < 3; ++k) {
            int N = m->nn[k * 192 + i];
            if (N < 0 || N >= 180) return CS3D_E_ARG;
            t->r0[k * 192 + i] = f3mag(X[i] - X[N], Y[i] - Y[N], Z[i] - Z[N]);
        }
    for (int n = 0; n < 180; n++) {
        float px = X[n], py = Y[n], pz = Z[n];
        int a = m->nn[n], b = m->nn[192 + n], c = m->nn[384 + n];
        float ix = X[a] - px, iy = Y[a] - py, iz = Z[a] - pz;
        float jx = X[b] - px, jy = Y[b] - py, jz = Z[b] - pz;
        float kx = X[c] - px, ky = Y[c] - py, kz = Z[c] - pz;
        float dij = ix * jx + iy * jy + iz * jz;
        float djk = jx * kx + jy * ky + jz * kz;
        float dik = ix * kx + iy * ky + iz * kz;
        t->theta0[3 * n + 0] = acosf(dij / (f3mag(ix, iy, iz) * f3mag(jx, jy, jz)));
        t->theta0[3 * n + 1] = acosf(djk / (f3mag(jx, jy, jz) * f3mag(kx, ky, kz)));
        t->theta0[3 * n + 2] = acosf(dik / (f3mag(ix, iy, iz) * f3mag(kx, ky, kz)));
    }
    return CS3D_OK;
}

// RANMAR, src/marsaglia.h:54-144.
int cs3d_rng_init(cs3d_rng *r, int ij, int kl)
{
    if (!r) return CS3D_E_ARG;
    if (ij < 0 || ij > 31328 || kl < 0 || kl > 30081) return CS3D_E_ARG;
    int i = (ij / 177) % 177 + 2;
    int j = ij % 177 + 2;
    int k = (kl / 169) % 178 + 1;
    int l = kl % 169;
    memset(r, 0, sizeof *r);
    for (int ii = 1; ii <= 97; ii++) {
        float s = 0.0f, t = 0.5f;
        for (int jj = 1; jj <= 24; jj++) {
            int mm = (((i * j) % 179) * k) % 179;
            i = j; j = k; k = mm;
            l = (53 * l + 1) % 169;
            if ((l * mm) % 64 >= 32) s += t;
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
    return CS3D_OK;
}

int cs3d_rng_draw(cs3d_rng *r, float *out, int len)
{
    if (!r || !r->ok || (len > 0 && !out)) return CS3D_E_ARG;
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
    return CS3D_OK;
}

int cs3d_rng_random_vector(cs3d_rng *r, float n[3])
{
    if (!r || !r->ok || !n) return CS3D_E_ARG;
    float ran2[2];
    float s;
    do {
        cs3d_rng_draw(r, ran2, 2);
        ran2[0] = 2.0f * ran2[0] - 1.0f;
        ran2[1] = 2.0f * ran2[1] - 1.0f;
        s = ran2[0] * ran2[0] + ran2[1] * ran2[1];
    } while (s >= 1.0f);
    float x1 = ran2[0], x2 = ran2[1];
    n[0] = 2 * x1 * sqrtf(1 - x1 * x1 - x2 * x2);
    n[1] = 2 * x2 * sqrtf(1 - x1 * x1 - x2 * x2);
    n[2] = 1 - 2 * (x1 * x1 + x2 * x2);
    return CS3D_OK;
}

// Centre of mass of one cell as the device computes it: six groups of 32
// slots (180..191 zero), each reduced pairwise in double, the group sums
// added in order, divided by 180 and rounded to float.
static float cell_mean(const float *v)
{
    double tot = 0.0;
    for (int g = 0; g < 6; ++g) {
        double w[32];
        for (int l = 0; l < 32; ++l) w[l] = 32 * g + l < 180 ? (double)v[32 * g + l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            double t[32];
            for (int l = 0; l < 32; ++l) t[l] = w[l] + w[l ^ o];
            memcpy(w, t, sizeof w);
        }
        tot += w[0];
    }
    return (float)(tot / 180.0);
}

// src/GPUbounce.cu:616-692.  The reference takes the centres of mass from
// its CenterOfMass kernel (float tree sum); they come from cell_mean here,
// the centre of mass of every other use in this library.
int cs3d_initial_stiffness(const cs3d_config *cfg, int n, const float *X, const float *Y, const float *Z,
                           cs3d_rng *rng, float *youngs)
{
    if (!cfg || n < 0 || (n && !youngs)) return CS3D_E_ARG;
    const float stiffness1 = cfg->stiff_factor1 * cfg->youngs_mod;
    const float stiffness2 = cfg->soft_stiff_factor * cfg->youngs_mod;
    for (int i = 0; i < n; ++i) youngs[i] = stiffness1;
    if (!cfg->use_different_stiffnesses || n == 0) return CS3D_OK;
    const float close = cfg->closeness_to_center;
    if (close > 0.f && close < 1.f) {
        if (!X || !Y || !Z) return CS3D_E_ARG;
        std::vector<float> cx(n), cy(n), cz(n);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        for (int i = 0; i < n; ++i) {
            cx[i] = cell_mean(X + (size_t)i * 192);
            cy[i] = cell_mean(Y + (size_t)i * 192);
            cz[i] = cell_mean(Z + (size_t)i * 192);
            sx = sx + cx[i];
            sy = sy + cy[i];
            sz = sz + cz[i];
        }
        // float3 / float is (1/a) * b, inc/VectorFunctions.hpp:84-92
        const float inv = 1.0f / (float)n;
        sx = inv * sx;
        sy = inv * sy;
        sz = inv * sz;
        std::vector<float> mags(n);
        float rmax = 0.f;
        for (int i = 0; i < n; ++i) {
            const float dx = cx[i] - sx, dy = cy[i] - sy, dz = cz[i] - sz;
            mags[i] = sqrtf(dx * dx + dy * dy + dz * dz);
            rmax = std::max(rmax, mags[i]);
        }
        for (int i = 0; i < n; ++i)
            if (mags[i] / rmax <= close) youngs[i] = stiffness2;
        return CS3D_OK;
    }
    int count = cfg->number_of_softer_cells;
    const float frac = cfg->fraction_of_softer_cells;
    if (frac > 0.f && frac < 1.f) count = (int)roundf(frac * (float)n);
    if (count > n) return CS3D_E_CONFIG;
    if (cfg->use_rigid_box) {
        for (int i = 0; i < count; ++i) youngs[i] = stiffness2;
        return CS3D_OK;
    }
    if (!rng || !rng->ok) return CS3D_E_ARG;
    for (int i = 0; i < count; ++i) {
        float u;
        cs3d_rng_draw(rng, &u, 1);
        const int ind = (int)roundf(u * (float)n);
        // ind == n names the next free slot, which a division overwrites before
        // any use (src/GPUbounce.cu:1257-1261)
        if (ind < n) youngs[ind] = stiffness2;
    }
    return CS3D_OK;
}

// initialize_C180s, src/GPUbounce.cu:1598-1774.
int cs3d_init_positions(const cs3d_config *cfg, const cs3d_mesh *mesh, int N, cs3d_rng *rng,
                        float *X, float *Y, float *Z)
{
    if (!cfg || !mesh || !X || !Y || !Z || N < 0) return CS3D_E_ARG;
    float initx[180], inity[180], initz[180];
    for (int a = 0; a < 180; ++a) { initx[a] = mesh->xyz[3 * a]; inity[a] = mesh->xyz[3 * a + 1]; initz[a] = mesh->xyz[3 * a + 2]; }
    float sumx = 0, sumy = 0, sumz = 0;
    for (int i = 0; i < 180; ++i) { sumx += initx[i]; sumy += inity[i]; sumz += initz[i]; }
    sumx = (float)(sumx / 180.0);
    sumy = (float)(sumy / 180.0);
    sumz = (float)(sumz / 180.0);
    for (int i = 0; i < 180; ++i) { initx[i] -= sumx; inity[i] -= sumy; initz[i] -= sumz; }
    memset(X, 0, sizeof(float) * 192 * (size_t)N);
    memset(Y, 0, sizeof(float) * 192 * (size_t)N);
    memset(Z, 0, sizeof(float) * 192 * (size_t)N);
    const float L1 = 3.0f;
    int side = (int)(sqrt((double)N) + 0.5);
    const float bx = cfg->box_len[0], by = cfg->box_len[1], bz = cfg->box_len[2];
    if (cfg->use_rigid_box) {
        float rCheck = powf((float)(0.75 * (1.f / 3.14159) * 0.786), 1.f / 3.f);
        float vol = bx * by * bz;
        int k = (int)floor(vol / 0.786);
        if (k < N) return CS3D_E_CONFIG;  // "Simulation box is too small", exit code 27
        if (cfg->rand_pos) {
            if (!rng || !rng->ok) return CS3D_E_ARG;
            std::vector<float> cx(N), cy(N), cz(N);
            int c = 0;
            float rands[3];
            long guard = 0;
            while (c < N) {
                if (++guard > 200000000L) return CS3D_E_CONFIG;
                cs3d_rng_draw(rng, rands, 3);
                float CMx = rands[0] * (bx - 1.f) + 1.f;
                float CMy = rands[1] * (by - 1.f) + 1.f;
                float CMz = cfg->flatbox ? bz / 2 : rands[2] * (bz - 1.f) + 1.f;
                bool far_enough = !(CMx + rCheck > bx || CMy + rCheck > by || CMz + rCheck > bz);
                for (int q = 0; q < c && far_enough; ++q)
                    if (f3mag(cx[q] - CMx, cy[q] - CMy, cz[q] - CMz) < 2 * rCheck) far_enough = false;
                if (far_enough) { cx[c] = CMx; cy[c] = CMy; cz[c] = CMz; ++c; }
            }
            for (int ci = 0; ci < N; ++ci)
                for (int a = 0; a < 180; ++a) {
                    X[ci * 192 + a] = initx[a] + cx[ci];
                    Y[ci * 192 + a] = inity[a] + cy[ci];
                    Z[ci * 192 + a] = initz[a] + cz[ci];
                }
        } else {
            float centerx = 0.5f * bx, centery = 0.5f * by, centerz = 0.5f * bz;
            for (int r = 0; r < N; ++r) {
                int ey = r % side, ex = r / side;
                for (int a = 0; a < 180; ++a) {
                    X[r * 192 + a] = (float)((double)(initx[a] + L1 * ex) + 0.5 * L1 + centerx);
                    Y[r * 192 + a] = (float)((double)(inity[a] + L1 * ey) + 0.5 * L1 + centery);
                    Z[r * 192 + a] = initz[a] + centerz;
                }
            }
        }
    } else {
        for (int r = 0; r < N; ++r) {
            int ey = r % side, ex = r / side;
            for (int a = 0; a < 180; ++a) {
                X[r * 192 + a] = (float)((double)(initx[a] + L1 * ex) + 0.5 * L1);
                Y[r * 192 + a] = (float)((double)(inity[a] + L1 * ey) + 0.5 * L1);
                Z[r * 192 + a] = initz[a] + cfg->z_offset;
            }
        }
    }
    return CS3D_OK;
}

// Binary trajectory, src/GPUbounce.cu:1007-1018, :2446-2477, :1508-1511.
struct cs3d_traj {
    FILE *f;
    int variable_stiffness;
};

int cs3d_traj_open(const char *path, int max_cells, int variable_stiffness, int max_frames,
                   cs3d_traj **out)
{
    if (!path || !out) return CS3D_E_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return CS3D_E_IO;
    int32_t h[3] = {max_cells, variable_stiffness, max_frames};
    if (fwrite(h, 4, 3, f) != 3) { fclose(f); return CS3D_E_IO; }
    cs3d_traj *t = new cs3d_traj{f, variable_stiffness};
    *out = t;
    return CS3D_OK;
}

int cs3d_traj_write_frame(cs3d_traj *t, int step, int frame, int n, const float *X,
                          const float *Y, const float *Z, const int32_t *types)
{
    if (!t || !t->f || n < 0 || (n > 0 && (!X || !Y || !Z))) return CS3D_E_ARG;
    int32_t h[3] = {step, frame, n};
    if (fwrite(h, 4, 3, t->f) != 3) return CS3D_E_IO;
    for (int32_t c = 0; c < n; ++c) {
        if (fwrite(&c, 4, 1, t->f) != 1) return CS3D_E_IO;
        if (fwrite(X + (size_t)c * 192, 4, 192, t->f) != 192) return CS3D_E_IO;
        if (fwrite(Y + (size_t)c * 192, 4, 192, t->f) != 192) return CS3D_E_IO;
        if (fwrite(Z + (size_t)c * 192, 4, 192, t->f) != 192) return CS3D_E_IO;
        if (t->variable_stiffness) {
            int32_t ty = types ? types[c] : 0;
            if (fwrite(&ty, 4, 1, t->f) != 1) return CS3D_E_IO;
        }
    }
    return CS3D_OK;
}

int cs3d_traj_close(cs3d_traj *t, int final_cells)
{
    if (!t) return CS3D_E_ARG;
    int rc = CS3D_OK;
    if (t->f) {
        if (final_cells >= 0) {
            int32_t v = final_cells;
            if (fseek(t->f, 0, SEEK_SET) != 0 || fwrite(&v, 4, 1, t->f) != 1) rc = CS3D_E_IO;
        }
        fclose(t->f);
    }
    delete t;
    return rc;
}

}  // extern "C"
