/*
 * ref_tree.cpp -- runs the reference's own tree build, multipoles and walk
 * (src/tree.cpp: refine :122-196, compute_multipoles, kick_fmm :384-635)
 * with its own particle store (src/part_vect.cpp) and kernels
 * (src/gravity.cpp), all compiled where they lie by oracle/Makefile (target
 * `reftree`) against the serial HPX stand-in oracle/hpx_shim.  TEST
 * INFRASTRUCTURE ONLY: it pins the oracle's restated tree and walk
 * (tg_oracle.cpp) to the reference's code.  Output goes to oracle/_ref/.
 *
 * One call = the reference's solve_gravity (src/main.cpp:31-73) on a fresh
 * tree built as its main loop builds it (src/main.cpp:201-207): refine until
 * no node splits, compute_multipoles(rung 0, output on), kick_fmm from the
 * root check item, then part_vect_kick_return.  Every particle is an output
 * particle, so the kick's output records carry each particle's FP32 phi and
 * g; the particle's input index travels in its group field (groups are off).
 * The kernels cache the options of their first call (src/gravity.cpp:
 * 176-187): one library copy per parameter set.  With `record`, every kernel
 * call of the walk is recorded (below) for comparison with the oracle's lists.
 */
#include <tigergrav/cosmo.hpp>
#include <tigergrav/gravity.hpp>
#include <tigergrav/groups.hpp>
#include <tigergrav/load.hpp>
#include <tigergrav/map.hpp>
#include <tigergrav/options.hpp>
#include <tigergrav/part_vect.hpp>
#include <tigergrav/tree.hpp>

#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

options options::global;
options &options::get() { return global; }
void options::set(options o) { global = o; }

/* the particle set part_vect_init loads (initialize.hpp): the caller's positions */
static std::vector<particle> g_init;
part_vect initial_particle_set(std::string, int, int) { return g_init; }

/* sky maps are off (opts.map): src/map.cpp (HEALPix, Silo) is not built,
 * and this is never reached */
void map_add_particle(const vect<double> &, double, double) { std::abort(); }

/*
 * The reference's interaction lists as its walk hands them to the kernels:
 * tree.cpp is compiled with each gravity_XX_yy renamed to reftree_XX_yy (the
 * Makefile's -D flags), so every kernel call of kick_fmm lands here, is
 * recorded (the sink: its first particle, or the node centre; the sources in
 * call order: particle positions, or multipole centres) and passed on to the
 * reference's kernel.  Kinds as the oracle numbers its lists: CC_D 0, CP_D 1,
 * CC_E 2, CP_E 3, PC_D 4, PP_D 5, PC_E 6, PP_E 7.
 */
struct CallRec {
    int kind;
    int32_t sink[3];
    int64_t nsink;
    std::vector<int32_t> src; /* 3 per source */
};
static std::vector<CallRec> g_calls;
static bool g_record = false;

template <class V>
static void rec_pos(int kind, const int32_t *sink, int64_t nsink, const V &y) {
    if (!g_record) return;
    CallRec r{kind, {sink[0], sink[1], sink[2]}, nsink, {}};
    r.src.reserve(3 * y.size());
    for (const auto &p : y)
        for (int d = 0; d < 3; d++) r.src.push_back(p[d]);
    g_calls.push_back(std::move(r));
}
static void rec_multi(int kind, const int32_t *sink, int64_t nsink, const std::vector<multi_src> &y) {
    if (!g_record) return;
    CallRec r{kind, {sink[0], sink[1], sink[2]}, nsink, {}};
    r.src.reserve(3 * y.size());
    for (const auto &m : y)
        for (int d = 0; d < 3; d++) r.src.push_back(m.x[d]);
    g_calls.push_back(std::move(r));
}
static void first_of(const std::vector<vect<pos_type>> &x, int32_t *s) {
    for (int d = 0; d < 3; d++) s[d] = x.empty() ? 0 : x[0][d];
}
static void of(const vect<pos_type> &x, int32_t *s) {
    for (int d = 0; d < 3; d++) s[d] = x[d];
}

std::uint64_t reftree_PP_direct(std::vector<force> &f, const std::vector<vect<pos_type>> &x,
                                std::vector<vect<pos_type>> y, bool do_phi) {
    int32_t s[3];
    first_of(x, s);
    rec_pos(5, s, (int64_t)x.size(), y);
    return gravity_PP_direct(f, x, std::move(y), do_phi);
}
std::uint64_t reftree_PP_ewald(std::vector<force> &f, const std::vector<vect<pos_type>> &x,
                               std::vector<vect<pos_type>> y) {
    int32_t s[3];
    first_of(x, s);
    rec_pos(7, s, (int64_t)x.size(), y);
    return gravity_PP_ewald(f, x, std::move(y));
}
std::uint64_t reftree_PC_direct(std::vector<force> &f, const std::vector<vect<pos_type>> &x,
                                std::vector<multi_src> &y) {
    int32_t s[3];
    first_of(x, s);
    rec_multi(4, s, (int64_t)x.size(), y);
    return gravity_PC_direct(f, x, y);
}
std::uint64_t reftree_PC_ewald(std::vector<force> &f, const std::vector<vect<pos_type>> &x,
                               std::vector<multi_src> &y) {
    int32_t s[3];
    first_of(x, s);
    rec_multi(6, s, (int64_t)x.size(), y);
    return gravity_PC_ewald(f, x, y);
}
std::uint64_t reftree_CC_direct(expansion<double> &L, const vect<pos_type> &x, std::vector<multi_src> &y) {
    int32_t s[3];
    of(x, s);
    rec_multi(0, s, 1, y);
    return gravity_CC_direct(L, x, y);
}
std::uint64_t reftree_CC_ewald(expansion<double> &L, const vect<pos_type> &x, std::vector<multi_src> &y) {
    int32_t s[3];
    of(x, s);
    rec_multi(2, s, 1, y);
    return gravity_CC_ewald(L, x, y);
}
std::uint64_t reftree_CP_direct(expansion<double> &L, const vect<pos_type> &x, std::vector<vect<pos_type>> y) {
    int32_t s[3];
    of(x, s);
    rec_pos(1, s, 1, y);
    return gravity_CP_direct(L, x, std::move(y));
}
std::uint64_t reftree_CP_ewald(expansion<double> &L, const vect<pos_type> &x, std::vector<vect<pos_type>> y) {
    int32_t s[3];
    of(x, s);
    rec_pos(3, s, 1, y);
    return gravity_CP_ewald(L, x, std::move(y));
}

/* the recorded calls of the last solve: count, then per call its kind, sink
 * (first particle or node centre), sink count and sources */
extern "C" int64_t reftree_num_calls() { return (int64_t)g_calls.size(); }
extern "C" int64_t reftree_call_size(int64_t k) {
    return k < 0 || k >= (int64_t)g_calls.size() ? -1 : (int64_t)g_calls[(size_t)k].src.size() / 3;
}
extern "C" int reftree_get_call(int64_t k, int32_t *kind, int32_t *sink, int64_t *nsink, int32_t *src) {
    if (k < 0 || k >= (int64_t)g_calls.size()) return -1;
    const CallRec &r = g_calls[(size_t)k];
    *kind = r.kind;
    for (int d = 0; d < 3; d++) sink[d] = r.sink[d];
    *nsink = r.nsink;
    std::memcpy(src, r.src.data(), sizeof(int32_t) * r.src.size());
    return 0;
}

/*
 * The reference's cosmology (src/cosmo.cpp, compiled into this library):
 * cosmos::advance_to_time on a given state, and the sequence of
 * cosmo_advance steps with the factors it leaves behind (the scale factors
 * of cosmo_scale, the float time, kick_dt1 / kick_dt2 per rung and the drift
 * factor).  cosmo_advance's rung steps use rung_to_dt, whose t_max the
 * reference caches on first use (tigergrav/time.hpp): this library's solves
 * and these calls all use t_max = 1.
 */
extern double kick_dt1[RUNG_MAX + 1];
extern double kick_dt2[RUNG_MAX + 1];
extern float this_time;
extern double drift_dt;

static void cosmo_options(double H0, double omega_m, double omega_lambda, int cosmic) {
    options o = options::get();
    o.H0 = H0;
    o.omega_m = omega_m;
    o.omega_lambda = omega_lambda;
    o.cosmic = cosmic != 0;
    o.t_max = 1.0;
    options::set(o);
}

/* out: a, adot, tau, drift_dt, kick_dt after advance_to_time(t0) from (a, adot, tau) */
extern "C" void reftree_cosmos_advance(double a, double adot, double tau, double t0, double H0, double omega_m,
                                       double omega_lambda, double *out) {
    cosmo_options(H0, omega_m, omega_lambda, 1);
    cosmos c(a, adot, tau);
    c.advance_to_time(t0);
    out[0] = c.get_scale();
    out[1] = c.get_Hubble() * c.get_scale();
    out[2] = c.get_tau();
    out[3] = c.get_drift_dt();
    out[4] = c.get_kick_dt();
}

/* cosmo_init(a0, adot0) with the reference's starting values (its globals as
 * a fresh run has them: kick_dt1 = kick_dt2 = {-1, 0, ...}, time 0, drift 0),
 * then one cosmo_advance per dt; per step out holds 5 + 2 (RUNG_MAX + 1) doubles:
 * the scale factor before and after (cosmo_scale), the float time, tau,
 * drift_dt, then kick_dt1[0..RUNG_MAX] and kick_dt2[0..RUNG_MAX] */
extern "C" int reftree_cosmo_steps(double a0, double adot0, double H0, double omega_m, double omega_lambda,
                                   const double *dts, int nsteps, double *out) {
    cosmo_options(H0, omega_m, omega_lambda, 1);
    for (int i = 0; i <= RUNG_MAX; i++) kick_dt1[i] = kick_dt2[i] = 0.0;
    kick_dt1[0] = kick_dt2[0] = -1.0;
    this_time = 0.0f;
    drift_dt = 0.0;
    cosmo_init(a0, adot0);
    const int W = 5 + 2 * (RUNG_MAX + 1);
    for (int k = 0; k < nsteps; k++) {
        cosmo_advance(dts[k]);
        double *o = out + (size_t)k * W;
        const auto sc = cosmo_scale();
        o[0] = sc.first;
        o[1] = sc.second;
        o[2] = this_time;
        o[3] = cosmo_time();
        o[4] = cosmo_drift_dt();
        for (int i = 0; i <= RUNG_MAX; i++) {
            o[5 + i] = cosmo_kick_dt1((rung_type)i);
            o[5 + RUNG_MAX + 1 + i] = cosmo_kick_dt2((rung_type)i);
        }
    }
    return 0;
}

/* the kick's output records are kept between calls by the reference
 * (kick_rc); the driver reads them after each solve and clears them */
extern kick_return kick_rc;

/*
 * The reference's rung kick and drift on given particles (src/part_vect.cpp:
 * part_vect_kick :341-436, part_vect_drift :493-540), with forces the caller
 * supplies: the particle store is loaded as part_vect_init loads it, the
 * call runs, and the store is read back (part_vect_read).  No cosmology, no
 * glass, Ewald off (so the second half-kick is the plain 0.5 dt).  t_max = 1.
 * part_vect_drift caches its options on first use: one parameter set per
 * library copy.
 */
static void load_particles(const int32_t *x, const float *v, const int8_t *rung, int64_t n, double dt_max,
                           double eta, double soft_len, double G) {
    options o = options();
    o.problem = "caller";
    o.problem_size = (std::uint64_t)n;
    o.out_parts = (int)n;
    o.m_tot = 1.0;
    o.G = G;
    o.dt_max = dt_max;
    o.eta = eta;
    o.soft_len = soft_len;
    o.t_max = 1.0;
    o.theta = 0.7;
    o.parts_per_node = 64;
    o.ewald = false;
    o.cosmic = false;
    o.glass = false;
    o.groups = false;
    o.map = false;
    options::set(o);
    g_init.assign((size_t)n, particle());
    for (int64_t i = 0; i < n; i++) {
        particle &p = g_init[(size_t)i];
        for (int d = 0; d < 3; d++) {
            p.x[d] = x[3 * i + d];
            p.v[d] = v[3 * i + d];
        }
        p.flags.out = 1;
        p.flags.rung = rung ? (std::uint64_t)rung[i] : 0;
        p.flags.group = (std::uint64_t)i;
    }
    cosmo_init(1.0, 0.0);
    part_vect_init();
}

/* part_vect_kick(0, n, min_rung, do_out, f) with f = g of the particles it
 * takes (rung >= min_rung, or all with do_out), in order; v, rungs and the
 * largest new rung out */
extern "C" int reftree_kick(const int32_t *x, const float *v, const int8_t *rung, const float *g, int64_t n,
                            int min_rung, int do_out, double dt_max, double eta, double soft_len, double G,
                            float *v_out, int8_t *rung_out, int32_t *max_rung) {
    load_particles(x, v, rung, n, dt_max, eta, soft_len, G);
    std::vector<force> f;
    for (int64_t i = 0; i < n; i++)
        if (rung[i] >= min_rung || do_out) {
            force q;
            q.phi = 0.0f;
            for (int d = 0; d < 3; d++) q.g[d] = g[3 * i + d];
            f.push_back(q);
        }
    kick_rc.out.clear();
    kick_rc.rung = 0;
    part_vect_kick(0, (part_iter)n, (rung_type)min_rung, do_out != 0, std::move(f)).get();
    *max_rung = kick_rc.rung;
    kick_rc.out.clear();
    const std::vector<particle> ps = part_vect_read(0, (part_iter)n).get();
    for (int64_t i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) v_out[3 * i + d] = ps[(size_t)i].v[d];
        rung_out[i] = (int8_t)ps[(size_t)i].flags.rung;
    }
    return 0;
}

/*
 * The reference's friends-of-friends partition (src/main.cpp:36-47 in
 * solve_gravity): a tree refined as for a solve, compute_multipoles, then
 * groups_reset, part_vect_init_groups, tree::find_groups from the root at
 * theta 0.99 and groups_execute_finders until nothing changes.  label[i] is
 * the reference's group id of caller particle i (its smallest storage index
 * in the tree's order), -1 without friends.  Positions must be distinct.
 * part_vect_find_groups caches the linking length on first use: one
 * parameter set per library copy.
 */
extern std::unordered_map<std::uint64_t, group> map[1024]; /* groups.cpp's catalogue, NMAP buckets */
extern "C" int reftree_fof_catalog(const int32_t *x, const float *v, int64_t n, double link_len, int leaf_max,
                                   int64_t *label, int64_t cap, double *cat, int64_t *ngroups);
extern "C" int reftree_fof(const int32_t *x, int64_t n, double link_len, int leaf_max, int64_t *label) {
    return reftree_fof_catalog(x, nullptr, n, link_len, leaf_max, label, 0, nullptr, nullptr);
}

/* the groups' catalogue of groups.cpp (the kick's groups_add_particle1 for
 * every grouped particle, groups_finish1, part_vect_find_groups2,
 * groups_finish2; src/main.cpp:56-66), after the partition above: per group
 * (up to cap) 13 doubles in cat -- its id, N, centre (3), v (3), dv (3),
 * rmax, rc; *ngroups = their number (velocities from v, which may be NULL) */
extern "C" int reftree_fof_catalog(const int32_t *x, const float *v, int64_t n, double link_len, int leaf_max,
                                   int64_t *label, int64_t cap, double *cat, int64_t *ngroups) {
    options o = options();
    o.problem = "caller";
    o.problem_size = (std::uint64_t)n;
    o.out_parts = (int)n;
    o.m_tot = 1.0;
    o.G = 1.0;
    o.theta = 0.7;
    o.parts_per_node = leaf_max;
    o.link_len = link_len;
    o.soft_len = 0.02;
    o.t_max = 1.0;
    o.dt_max = 1.0 / 64.0;
    o.eta = 0.2;
    o.ewald = true;
    o.groups = true;
    o.cosmic = false;
    o.glass = false;
    o.map = false;
    o.workgroup_size = 32;
    o.oversubscription = 1;
    options::set(o);
    g_init.assign((size_t)n, particle());
    std::unordered_map<std::uint64_t, int64_t> index;
    auto key = [](const int32_t *p) {
        std::uint64_t h = 1469598103934665603ull;
        for (int d = 0; d < 3; d++) h = (h ^ (std::uint32_t)p[d]) * 1099511628211ull;
        return h;
    };
    for (int64_t i = 0; i < n; i++) {
        particle &p = g_init[(size_t)i];
        for (int d = 0; d < 3; d++) {
            p.x[d] = x[3 * i + d];
            p.v[d] = v ? v[3 * i + d] : 0.0f;
        }
        p.flags.out = 1;
        p.flags.rung = 0;
        p.flags.group = DEFAULT_GROUP;
        if (!index.emplace(key(x + 3 * i), i).second) return -2; /* positions (hashes) must be distinct */
    }
    cosmo_init(1.0, 0.0);
    part_vect_init();
    tree::set_theta(0.7);
    tree_client root = hpx::new_<tree>(hpx::find_here(), 1, 0, (part_iter)n, 0).get();
    refine_return rr;
    do {
        rr = root.refine(0);
    } while (rr.rc);
    root.compute_multipoles(0, false, 0);
    auto root_list = std::vector<check_item>(1, root.get_check_item());
    groups_reset();
    part_vect_init_groups();
    tree::set_theta(0.99);
    root.find_groups(root_list, 0);
    int rounds = 0;
    while (groups_execute_finders())
        if (++rounds > 100000) return -3;
    const std::vector<particle> ps = part_vect_read(0, (part_iter)n).get();
    for (const particle &p : ps) {
        const int32_t q[3] = {p.x[0], p.x[1], p.x[2]};
        const auto it = index.find(key(q));
        if (it == index.end()) return -4;
        label[it->second] = p.flags.group == DEFAULT_GROUP ? -1 : (int64_t)p.flags.group;
    }
    if (cat) {
        /* the output kick (zero forces: velocities stay) feeds groups_add_particle1 */
        std::vector<force> f((size_t)n);
        for (auto &q : f) {
            q.phi = 0.0f;
            q.g = vect<float>(0.0f);
        }
        kick_rc.out.clear();
        part_vect_kick(0, (part_iter)n, 0, true, std::move(f)).get();
        kick_rc.out.clear();
        groups_finish1();
        part_vect_find_groups2();
        groups_finish2();
        int64_t k = 0;
        for (int m = 0; m < 1024; m++)
            for (const auto &entry : map[m]) {
                if (k < cap) {
                    double *o = cat + 13 * k;
                    const group &gr = entry.second;
                    o[0] = (double)entry.first;
                    o[1] = (double)gr.N;
                    for (int d = 0; d < 3; d++) {
                        o[2 + d] = gr.x[d];
                        o[5 + d] = gr.v[d];
                        o[8 + d] = gr.dv[d];
                    }
                    o[11] = gr.rmax;
                    o[12] = gr.rc;
                }
                k++;
            }
        *ngroups = k;
    }
    groups_reset();
    hpx::release_components();
    return 0;
}

/* The reference's Gadget-1 reader (src/load.cpp:34-96, compiled into this
 * library with src/rand.cpp for its output flag): up to cap particles' int32
 * positions and float velocities of the file, *n their number. */
extern "C" int reftree_load_gadget1(const char *path, int64_t cap, int32_t *x, float *v, int64_t *n) {
    options o = options::get();
    o.out_parts = 0;
    o.problem_size = 1;
    options::set(o);
    const std::vector<particle> ps = load_particles(std::string(path));
    *n = (int64_t)ps.size();
    if (*n > cap) return -1;
    for (int64_t i = 0; i < *n; i++)
        for (int d = 0; d < 3; d++) {
            x[3 * i + d] = ps[(size_t)i].x[d];
            v[3 * i + d] = ps[(size_t)i].v[d];
        }
    return 0;
}

/* part_vect_drift(0, mrung): every particle moves by v rung_to_dt(mrung), wrapped into the box */
extern "C" int reftree_drift(const int32_t *x, const float *v, int64_t n, int mrung, int32_t *x_out) {
    load_particles(x, v, nullptr, n, 1.0, 0.2, 0.01, 1.0);
    part_vect_drift(0.0, (rung_type)mrung);
    const std::vector<particle> ps = part_vect_read(0, (part_iter)n).get();
    for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) x_out[3 * i + d] = ps[(size_t)i].x[d];
    return 0;
}

static bool g_inited = false;
static double g_key[7];

extern "C" int reftree_solve(const int32_t *x, int64_t n, double theta, int ewald, int leaf_max, double soft_len,
                             double G, int record, float *phi, float *g, uint64_t *istats, int64_t *tree_counts) {
    const double key[7] = {theta, (double)ewald, (double)leaf_max, soft_len, G, (double)n, 1.0};
    if (g_inited && std::memcmp(key, g_key, sizeof(key)) != 0) return -1; /* one parameter set per copy */
    options o = options();
    o.problem = "caller";
    o.problem_size = (std::uint64_t)n;
    o.out_parts = (int)n;
    o.theta = theta;
    o.ewald = ewald != 0;
    o.parts_per_node = leaf_max;
    o.soft_len = soft_len;
    o.m_tot = 1.0;
    o.G = G;
    o.gravity = true;
    o.solver_test = false;
    o.cosmic = false;
    o.glass = false;
    o.groups = false;
    o.map = false;
    o.balanced_tree = false;
    o.workgroup_size = 32;
    o.oversubscription = 1;
    o.dt_max = 1.0 / 64.0;
    o.t_max = 1.0;
    o.eta = 0.2;
    o.nout = 1;
    options::set(o);
    std::memcpy(g_key, key, sizeof(key));
    g_inited = true;

    g_init.assign((size_t)n, particle());
    for (int64_t i = 0; i < n; i++) {
        particle &p = g_init[(size_t)i];
        for (int d = 0; d < 3; d++) {
            p.x[d] = x[3 * i + d];
            p.v[d] = 0.0f;
        }
        p.flags.out = 1;
        p.flags.rung = 0;
        p.flags.group = (std::uint64_t)i;
    }
    cosmo_init(1.0, 0.0);
    part_vect_init();
    tree::set_theta(theta);
    tree_client root = hpx::new_<tree>(hpx::find_here(), 1, 0, (part_iter)n, 0).get();
    refine_return rr;
    do {
        rr = root.refine(0);
    } while (rr.rc);
    tree_counts[0] = (int64_t)rr.nodes;
    tree_counts[1] = (int64_t)rr.leaves;
    kick_rc.out.clear();
    kick_rc.rung = 0;
    kick_rc.stats.zero();
    g_calls.clear();
    g_record = record != 0;
    root.compute_multipoles(0, true, 0);
    auto root_list = std::vector<check_item>(1, root.get_check_item());
    expansion<double> L;
    L = 0.0;
    const interaction_stats st = root.kick_fmm(root_list, root_list, {{0.5, 0.5, 0.5}}, L, 0, true, 0);
    const kick_return rc = part_vect_kick_return();
    g_record = false;
    istats[0] = st.PP_direct;
    istats[1] = st.PP_ewald;
    istats[2] = st.CC_direct;
    istats[3] = st.CC_ewald;
    istats[4] = st.CP_direct;
    istats[5] = st.CP_ewald;
    int64_t seen = 0;
    for (const output &out : rc.out) {
        const std::uint64_t i = out.id;
        if (i >= (std::uint64_t)n) return -2;
        phi[i] = out.phi;
        for (int d = 0; d < 3; d++) g[3 * i + d] = out.g[d];
        seen++;
    }
    kick_rc.out.clear();
    hpx::release_components();
    return seen == n ? 0 : -3;
}
