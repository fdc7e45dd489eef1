/*
 * tigergrav_b200.h -- C ABI of the B200 periodic tree-gravity library
 * (tigergrav_b200/libtigergrav_b200.so).
 *
 * The library replaces TigerGrav's gravity evaluation path: the tree built by
 * tree::refine, the multipoles of tree::compute_multipoles, the dual-list walk
 * of tree::kick_fmm with the eight gravity_{PP,PC,CC,CP}_{direct,ewald}
 * kernels, L2L/L2P, and the kick/drift of the particle store.  All entry
 * points are plain C: pointers, sizes, an int status, and a CUDA stream
 * passed as `void *` (a cudaStream_t; NULL is the legacy default stream).
 *
 * Conventions
 *  - Positions are the reference's int32 fixed point, x = i * 2^-32 + 0.5
 *    (tigergrav/position.hpp:13-37), interleaved x,y,z per particle.
 *  - Velocities and forces are interleaved x,y,z per particle.
 *  - "where" arguments say whether a pointer is host (TG_HOST) or device
 *    (TG_DEVICE) memory; host buffers are copied through pinned staging.
 *  - Every call returns TG_OK (0) or a TG_ERR_* code; tg_error_string names it.
 *  - A handle is not thread-safe; distinct handles may be used concurrently.
 *  - Kernels never trap: bounded waits and capacity checks end in a status.
 */
#ifndef TIGERGRAV_B200_H
#define TIGERGRAV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum tg_status {
    TG_OK = 0,
    TG_ERR_ARG = 1,      /* bad argument (sizes, NULL pointers, NaN positions) */
    TG_ERR_CUDA = 2,     /* a CUDA runtime call failed */
    TG_ERR_CAPACITY = 3, /* a list buffer overflowed and the retry limit was hit */
    TG_ERR_DEPTH = 4,    /* more than leaf_max particles share a 63-level box */
    TG_ERR_TIMEOUT = 5,  /* a bounded device wait ran out */
    TG_ERR_STATE = 6,    /* call out of order (e.g. forces before a build) */
    TG_ERR_NOMEM = 7,    /* device allocation failed */
    TG_ERR_SIZE = 8      /* n above what tg_energy_noalloc's fixed scratch holds */
};

enum tg_precision {
    TG_PREC_F32 = 0, /* FP32 interaction arithmetic, per-leaf compensated (Kahan) sums */
    TG_PREC_F64 = 1  /* plain FP64 port: all interaction arithmetic in double */
};

enum tg_where { TG_HOST = 0, TG_DEVICE = 1 };

/* Interaction-list kinds, CSR per node.  The first four are built at every
 * node (tree.cpp:424-494), the last four at leaves (tree.cpp:530-629). */
enum tg_list_kind {
    TG_CC_D = 0, TG_CP_D = 1, TG_CC_E = 2, TG_CP_E = 3,
    TG_PC_D = 4, TG_PP_D = 5, TG_PC_E = 6, TG_PP_E = 7
};

/* Solver parameters.  Replaces the reference's global options object
 * (tigergrav/options.hpp:5-82) for the fields the gravity path reads. */
typedef struct tg_params {
    double theta;      /* opening angle; tree::set_theta (src/tree.cpp:93-111) */
    double soft_len;   /* h, GADGET spline softening length (options::soft_len) */
    double m;          /* particle mass, m_tot / problem_size (src/gravity.cpp:186) */
    double G;          /* gravitational constant (options::G) */
    int32_t ewald;     /* 1: periodic box with Ewald correction (options::ewald) */
    int32_t leaf_max;  /* parts_per_node, 1..128 (src/options.cpp:52) */
    int32_t precision; /* tg_precision */
    int32_t device;    /* CUDA device ordinal */
} tg_params;

typedef struct tg_stats {
    int64_t n;            /* particles */
    int64_t nodes;        /* tree nodes (including empty ones) */
    int64_t leaves;
    int32_t depth;        /* deepest level */
    int32_t walk_retries; /* list-buffer regrowths in the last walk */
    /* interaction_stats as the reference files them (tigergrav/tree.hpp:84-114):
     * PP_direct, PP_ewald, CC_direct, CC_ewald, CP_direct, CP_ewald
     * (leaf PC counts filed under CP, as src/tree.cpp:618,627 do) */
    uint64_t ref_stats[6];
    /* per-kind interaction counts: PP_D, PP_E, PC_D, PC_E (sink-source pairs),
     * CC_D, CC_E (node-node), CP_D, CP_E (node-particle) */
    uint64_t counts[8];
    double flops;         /* reference flop convention (src/gravity.cpp:299-784, tree.cpp:234) */
    /* device time of the last solve, per phase, milliseconds */
    double ms_build, ms_multipoles, ms_walk, ms_nodes, ms_leaves;
    double ms_kick_drift; /* the tg_kick_drift right before the last solve, if there was one */
    int64_t launches;     /* kernels of this library launched on this handle so far */
    double ms_pp;         /* part of ms_leaves spent in the FP32 PP-direct kernel (0 when it is not used) */
    int64_t device_bytes; /* device memory held by this library's buffers in the process (all handles) */
} tg_stats;

typedef struct tg_solver tg_solver;

const char *tg_error_string(int status);
/* library version string */
const char *tg_version(void);

/* ---- solver object -------------------------------------------------- */
/* Replaces options::process_options + tree::set_theta (src/options.cpp:28-94,
 * src/tree.cpp:93-111): validates and stores the parameters. */
int tg_create(const tg_params *params, tg_solver **out);
int tg_destroy(tg_solver *s);

/* Replaces part_vect_init (src/part_vect.cpp:654-673): loads n particles.
 * x: n*3 int32, v: n*3 float (NULL = zero velocities).  n < 1 or a non-finite
 * velocity gives TG_ERR_ARG (then no particles are loaded). */
int tg_set_particles(tg_solver *s, const int32_t *x, const float *v, int64_t n, int where, void *stream);
/* Positions / velocities in the caller's original particle order. */
int tg_get_particles(tg_solver *s, int32_t *x, float *v, int where, void *stream);

/* tree::refine iterated to completion (src/tree.cpp:122-201, src/main.cpp:171-175). */
int tg_build(tg_solver *s, void *stream);
/* tree::compute_multipoles (src/tree.cpp:203-296). */
int tg_multipoles(tg_solver *s, void *stream);
/* tree::kick_fmm list generation (src/tree.cpp:378-635).  The list pools are
 * sized from the tree, then from the totals of the last walk; a walk that
 * overflows a pool writes nothing out of bounds, regrows the pools to the
 * totals it asked for and runs again (stats.walk_retries counts the reruns). */
int tg_walk(tg_solver *s, void *stream);
/* First capacity (entries) of every list pool and of the walk's scratch for
 * the following walks, 0 = sized from the tree (the default).  A small value
 * forces the regrowth path; the lists it ends with are the same.  No
 * counterpart in the reference (its lists are std::vectors). */
int tg_set_walk_capacity(tg_solver *s, int64_t entries);
/* kick_fmm evaluation: CC/CP, L2L, L2P, PC/PP, direct and Ewald. */
int tg_forces(tg_solver *s, void *stream);
/* solve_gravity (src/main.cpp:31-73): build + multipoles + walk + forces. */
int tg_solve_gravity(tg_solver *s, void *stream);

/* Forces in the caller's order: phi[n], g[n*3] (either may be NULL). */
int tg_get_forces(tg_solver *s, float *phi, float *g, int where, void *stream);
int tg_get_forces_f64(tg_solver *s, double *phi, double *g, int where, void *stream);

/* Kick with the last forces: v += g * G * dt (part_vect_kick, src/part_vect.cpp:341-436,
 * as a plain fixed-dt half kick). */
int tg_kick(tg_solver *s, double dt, void *stream);
/* Drift x = wrap(x + v dt), requantised (part_vect_drift, src/part_vect.cpp:493-540). */
int tg_drift(tg_solver *s, double dt, void *stream);
/* FP64 reductions: out[0] = E_kin, out[1] = E_pot (0.5 m phi G), out[2..4] = sum v / n. */
int tg_energy(tg_solver *s, double out[5], void *stream);

/* The same reductions over caller-owned device arrays, allocating nothing:
 * for callers that cannot allocate device memory where they need the
 * reduction (a fixed memory arena handed to the library up front, an
 * allocation-free time loop).  No counterpart in the reference.
 * v: n*3 floats, phi: n floats (NULL: E_pot = 0), out: 5 doubles, all device
 * memory; n <= TG_NOALLOC_MAX_N, else TG_ERR_SIZE.  The partial sums live in a
 * fixed 2.5 MiB array inside the library, shared by every call: calls that
 * overlap on the GPU race.  The first call on a device looks the array up
 * (cudaGetSymbolAddress); make it before any stream capture.  The call runs
 * on `device` and leaves the calling thread's current device as it was. */
#define TG_NOALLOC_MAX_N (1ll << 26)
int tg_energy_noalloc(const float *v, const float *phi, int64_t n, double m, double G, double *out,
                      int device, void *stream);
/* The kick that closes one step, the kick that opens the next and the drift
 * between them in one pass over the particles: v += g G dt_close, v += g G
 * dt_open (each product rounded to float and added as tg_kick does; dt_close
 * = 0 skips the first), then x = wrap(x + v dt_drift) as tg_drift.  The
 * reference fuses its kick into the force stage (src/tree.cpp:630) and
 * drifts in a separate pass (part_vect_drift, src/part_vect.cpp:493-540).
 * Needs forces; like tg_drift it invalidates the tree. */
int tg_kick_drift(tg_solver *s, double dt_close, double dt_open, double dt_drift, void *stream);
/* n_steps kick-drift-kick leapfrog steps of dt (first call computes forces if
 * needed); between steps the closing and opening kicks and the drift run as
 * one tg_kick_drift, with the same arithmetic as kick, drift, solve, kick. */
int tg_leapfrog(tg_solver *s, double dt, int n_steps, void *stream);

/* ---- differentiation (forward/backward pair, like torch.autograd.Function) ----
 * No counterpart in the reference (its leapfrog, src/part_vect.cpp:341-540 driven
 * by src/main.cpp:258-273, is forward only).
 * tg_forward: n_steps leapfrog steps as tg_leapfrog, checkpointing positions and
 * velocities (caller order) before the first step and after each step.
 * tg_backward: given dL/dx and dL/dv after the last step (n x 3 doubles, caller
 * order; gv may be NULL for zero) returns dL/dx and dL/dv before the first step
 * (gv0 may be NULL).  Each step's Jacobian-vector product recomputes the tree,
 * multipoles and lists at that step's checkpoint; see tg_tidal for the terms.
 * Leaves the solver at the first checkpoint (tree and lists built, no forces).
 * tg_tidal: out = J u with J = dg/dx (g the accelerations per unit G) at the
 * current particles and lists (after tg_walk): far field through the local
 * expansion's tidal tensor, PC through the multipoles' (monopole + quadrupole)
 * tidal tensors, PP (direct and Ewald) through the exact pair Hessians acting
 * on u_i - u_j. */
int tg_forward(tg_solver *s, double dt, int n_steps, void *stream);
int tg_backward(tg_solver *s, const double *gx, const double *gv, double *gx0, double *gv0, int where, void *stream);
int tg_tidal(tg_solver *s, const double *u, double *out, int where, void *stream);

/* ---- cosmological kick and drift factors ----------------------------------
 * cosmos::advance_to_time / cosmo_advance (src/cosmo.cpp:50-106,187-218): the
 * Friedmann expansion a(t) with a'' = H0^2 (-omega_m / (2 a^2) + omega_lambda a),
 * integrated by the reference's fixed-step RK4.  state = {a, da/dt, tau}; one
 * call advances it by dt and returns factors = {int_t^{t+dt/2} dt'/a,
 * int_t^{t+dt} dt'/a^2, int_{t+dt/2}^{t+dt} dt'/a}: the first half kick, the
 * drift and the second half kick, to be passed as dt to tg_kick / tg_drift.
 * Host only (no GPU needed).  tg_leapfrog_cosmo runs n_steps such steps. */
typedef struct tg_cosmo_params {
    double H0;            /* Hubble constant in code units */
    double omega_m;
    double omega_lambda;
} tg_cosmo_params;
int tg_cosmo_kdk(const tg_cosmo_params *p, double *state, double dt, double *factors);
int tg_leapfrog_cosmo(tg_solver *s, const tg_cosmo_params *p, double *state, double dt, int n_steps, void *stream);

/* ---- initial conditions -----------------------------------------------------
 * load_header / load_particles (src/load.cpp:13-96): an N-GenIC / Gadget-1 file
 * (256-byte io_header_1, then positions and velocities of type-1 particles).
 * header (8 doubles, may be NULL): npart[1], redshift, mass[1], Omega0,
 * OmegaLambda, HubbleParam, BoxSize, time.  With x == NULL only the header and
 * *n_out are read; otherwise x (n x 3 int32, fixed point) and v (n x 3 float,
 * may be NULL) are filled as the reference does (shift by 0.5 N^(-1/3), wrap,
 * double_to_pos; v * a^1.5); capacity < n gives TG_ERR_SIZE.  Host only. */
int tg_load_gadget1(const char *path, double *header, int32_t *x, float *v, int64_t capacity, int64_t *n_out);

/* ---- friends-of-friends groups ----------------------------------------------
 * tree::find_groups + part_vect_find_groups (src/tree.cpp:637-759,
 * src/part_vect.cpp:85-124) and the group statistics of src/groups.cpp:124-226.
 * tg_find_groups: friends are particle pairs whose squared fixed-point
 * separation (int32 difference: nearest image) is below
 * ((uint64)(link_len n^(-1/3) (2^32-1)))^2 and non-zero; groups are the
 * connected components.  group (n int64, caller order, host or device per
 * where, may be NULL) receives each particle's group id -- the smallest caller
 * index in its group -- or -1 (the reference's DEFAULT_GROUP) for a particle
 * without friends; *ngroups (may be NULL) the number of groups.  Builds the
 * tree and multipoles when the handle has none; link_len n^(-1/3) must lie in
 * (0, 0.5).  Without ewald the separation is the plain difference.
 * tg_group_catalog: statistics of the groups of the last tg_find_groups on the
 * current tree (TG_ERR_STATE otherwise), ids ascending, 14 doubles per group:
 * id, N, centre x[3] (nearest-image mean, in [0,1)), mean v/a [3], velocity
 * dispersion [3] (rms of v/a - mean per axis), rmax, rc (median radius,
 * element N/2 of the sorted radii a |x - centre|), 0.  a: scale factor.  With
 * out == NULL only *ngroups is set; capacity < ngroups gives TG_ERR_SIZE. */
int tg_find_groups(tg_solver *s, double link_len, int64_t *group, int64_t *ngroups, int where, void *stream);
/* Hook attempts per union in tg_find_groups' lock-free union-find (default
 * 65536; 0 and up).  A union that runs out of attempts makes tg_find_groups
 * answer TG_ERR_TIMEOUT instead of spinning; a small limit injects that fault
 * from the host.  No counterpart in the reference (serial label propagation). */
int tg_set_fof_retry_limit(tg_solver *s, int32_t tries);

/* ---- hierarchical (rung) time steps ------------------------------------------
 * tigergrav/time.hpp:12-48, the main loop step (src/main.cpp:266-313) and the
 * rung kick of part_vect_kick (src/part_vect.cpp:340-381).  Rung r has step
 * t_max / 2^r; the integer time itime counts t_max / 2^31.  tg_rung_step with
 * max_rung < 0 (a fresh state: itime 0) does the first solve and kick; each
 * later call drifts all particles by t_max / 2^max_rung, advances itime by
 * 2^(31 - max_rung), solves gravity with only the particles of rung >=
 * min_rung(itime) as sinks (all particles when all_forces; the reference's
 * do_out) and kicks those: half a step of the old rung (not on rung 0), new
 * rung from dt = min(dt_max, eta sqrt(soft_len / 2.8 / |g G|)) (at least
 * min_rung), half a step of the new rung; stored rung max(rung, old - 1, 1).
 * max_rung returns the largest new rung of the active particles.  Non-
 * cosmological; the second half kick is 0.5 dt (the reference's periodic
 * runs zero it by testing opts.ewald for opts.cosmic).  Forces of inactive
 * particles are not evaluated and the lists hold active sinks only, so after
 * a step without all_forces tg_forces, tg_get_forces, tg_tidal and tg_get_list
 * answer TG_ERR_STATE until the next full solve.  Rungs start at 0
 * (tg_set_particles) and travel with the particles; tg_get_rungs reads them in
 * caller order (n int8).  On an error *state is left as it was, and so are the
 * velocities and rungs (a rung overflow is found before any kick is applied);
 * the positions may have drifted. */
typedef struct {
    double t_max;  /* options::t_max */
    double dt_max; /* options::dt_max */
    double eta;    /* options::eta */
} tg_rung_params;
typedef struct {
    uint32_t itime;     /* integer time, 2^31 == t_max */
    int32_t max_rung;   /* largest rung of the last kick; -1 before the first step */
    int32_t min_rung;   /* lowest active rung of the last step */
    int32_t reserved;
    int64_t num_active; /* particles kicked by the last step */
    double t;           /* itime in units of time */
} tg_rung_state;
int tg_rung_step(tg_solver *s, const tg_rung_params *p, tg_rung_state *state, int all_forces, void *stream);
/* The same step with the reference's cosmological factors (opts.cosmic):
 * before the drift, cosmo_advance (src/cosmo.cpp:187-218) moves the expansion
 * by the step of the largest rung (time accumulated in float, as the
 * reference's this_time) and gives, per rung, kick_dt1 (back over half the
 * rung's step; kept from earlier steps until the time reaches the step) and
 * kick_dt2 (ahead over half the step), and the drift factor over the step.
 * The kick (src/part_vect.cpp:358-381) closes with kick_dt1 of the old rung,
 * chooses the rung from |g G| / a^3 with a the scale factor at the start of
 * the step, and opens with kick_dt2 of the stored rung (the fixed check:
 * opts.cosmic where the reference tests opts.ewald, src/part_vect.cpp:376).
 * tg_cosmo_rung_init starts a state at scale factor a and da/dt adot (the
 * reference starts at a = 1, adot = H0: cosmos::cosmos, src/cosmo.cpp:29-37).
 * *cs changes only when the step succeeds. */
typedef struct {
    double a, adot, tau; /* the expansion now (this_cosmos) */
    double a_last;       /* the scale factor at the start of the last step (last_cosmos) */
    float time;          /* the reference's float time accumulator (this_time) */
    int32_t reserved;
    double kick1[31];    /* kick_dt1 per rung, kept between steps like the reference's array */
} tg_cosmo_rung_state;
int tg_cosmo_rung_init(tg_cosmo_rung_state *cs, double a, double adot);
int tg_rung_step_cosmo(tg_solver *s, const tg_rung_params *p, tg_rung_state *state, const tg_cosmo_params *cp,
                       tg_cosmo_rung_state *cs, int all_forces, void *stream);
int tg_get_rungs(tg_solver *s, int8_t *rung, int where, void *stream);
int tg_group_catalog(tg_solver *s, double a, double *out, int64_t capacity, int64_t *ngroups, void *stream);

/* ---- batches of independent boxes ---------------------------------------
 * No counterpart in the reference (one box per run).  nboxes periodic unit
 * boxes, box b with counts[b] particles, its own m = 1/counts[b] and
 * soft_len = 0.02 counts[b]^(-1/3) (params->m and soft_len are ignored);
 * theta, G, ewald, leaf_max, precision and device come from params.  Particle
 * and force arrays are the boxes' arrays concatenated in box order.  Calls run
 * the boxes concurrently on nstreams streams (one host thread each) and return
 * when all are done.  tg_batch_autotune times one evaluation per box for each
 * candidate leaf size (1..128) and keeps the fastest per box (chosen: nboxes
 * ints, may be NULL). */
typedef struct tg_batch tg_batch;
int tg_batch_create(const tg_params *params, int32_t nboxes, const int64_t *counts, int32_t nstreams, tg_batch **out);
int tg_batch_destroy(tg_batch *b);
int64_t tg_batch_size(tg_batch *b);
int tg_batch_set_particles(tg_batch *b, const int32_t *x, const float *v, int where);
int tg_batch_autotune(tg_batch *b, const int32_t *leaf_sizes, int32_t nsizes, int32_t *chosen);
int tg_batch_solve(tg_batch *b);
int tg_batch_leapfrog(tg_batch *b, double dt, int n_steps);
int tg_batch_get_forces(tg_batch *b, float *phi, float *g, int where);

int tg_get_stats(tg_solver *s, tg_stats *out);
/* Device memory held by this handle's buffers: one "name bytes" line per
 * buffer and a "total" line, NUL-terminated, into buf (cap bytes; TG_ERR_SIZE
 * if it does not fit).  For planning runs against the 180 GB of one GPU; no
 * counterpart in the reference. */
int tg_memory_report(tg_solver *s, char *buf, int64_t cap);

/* ---- introspection (parity tests) ----------------------------------- */
int64_t tg_num_nodes(tg_solver *s);
/* Node arrays in host memory, level order; any pointer may be NULL.
 * boxid = 1 << level | Morton prefix (src/tree.cpp:159-160, src/range.cpp:134-168). */
int tg_get_nodes(tg_solver *s, uint64_t *boxid, int32_t *level, int64_t *pbegin, int64_t *pend,
                 int32_t *child0, int32_t *parent, int32_t *x, float *r, float *rmax, float *m);
/* perm[i] = caller index of the particle at sorted position i. */
int tg_get_perm(tg_solver *s, int64_t *perm);
int64_t tg_list_size(tg_solver *s, int kind);
/* CSR copy of list `kind`: offsets[num_nodes+1], ids[list_size] (host). */
int tg_get_list(tg_solver *s, int kind, int64_t *offsets, int32_t *ids);

/* ---- kernel-level seams (all pointers device memory) ------------------
 * The eight reference kernels (tigergrav/gravity.hpp:39-46) evaluated over
 * many sink groups at once.  Group k has sinks [sink_off[k], sink_off[k+1])
 * and sources [src_off[k], src_off[k+1]).  f is nsinks x 4 doubles
 * (phi, gx, gy, gz) and L is ngroups x 35 doubles; both accumulate with +=.
 * Multipole sources: src_m (17 floats each), src_x (3 int32 each).
 * CC/CP sinks: sink_x holds one position per group.
 * Parameters (h, m, ewald) come from params.  flops (may be NULL) receives
 * the reference's flop count (src/gravity.cpp:299,365,425,485,613,677,730,784). */
int tg_gravity_PP_direct(const tg_params *params, int64_t ngroups, const int64_t *sink_off,
                         const int32_t *sink_x, const int64_t *src_off, const int32_t *src_x,
                         double *f, int do_phi, uint64_t *flops, void *stream);
int tg_gravity_PP_ewald(const tg_params *params, int64_t ngroups, const int64_t *sink_off,
                        const int32_t *sink_x, const int64_t *src_off, const int32_t *src_x,
                        double *f, uint64_t *flops, void *stream);
int tg_gravity_PC_direct(const tg_params *params, int64_t ngroups, const int64_t *sink_off,
                         const int32_t *sink_x, const int64_t *src_off, const float *src_m,
                         const int32_t *src_x, double *f, uint64_t *flops, void *stream);
int tg_gravity_PC_ewald(const tg_params *params, int64_t ngroups, const int64_t *sink_off,
                        const int32_t *sink_x, const int64_t *src_off, const float *src_m,
                        const int32_t *src_x, double *f, uint64_t *flops, void *stream);
int tg_gravity_CC_direct(const tg_params *params, int64_t ngroups, const int32_t *sink_x,
                         const int64_t *src_off, const float *src_m, const int32_t *src_x,
                         double *L, uint64_t *flops, void *stream);
int tg_gravity_CC_ewald(const tg_params *params, int64_t ngroups, const int32_t *sink_x,
                        const int64_t *src_off, const float *src_m, const int32_t *src_x,
                        double *L, uint64_t *flops, void *stream);
int tg_gravity_CP_direct(const tg_params *params, int64_t ngroups, const int32_t *sink_x,
                         const int64_t *src_off, const int32_t *src_x, double *L,
                         uint64_t *flops, void *stream);
int tg_gravity_CP_ewald(const tg_params *params, int64_t ngroups, const int32_t *sink_x,
                        const int64_t *src_off, const int32_t *src_x, double *L,
                        uint64_t *flops, void *stream);

/* ---- measurement ------------------------------------------------------
 * FP64 direct Ewald sum (ground truth) at ns sample particles of the
 * current particle set: phi[ns], g[ns*3] in host memory.  alpha is the
 * Ewald split (>= 4.2); results are independent of it to ~1e-13. */
int tg_truth(tg_solver *s, const int64_t *samples, int64_t ns, double alpha, double *phi, double *g,
             void *stream);
/* Measured FP32 FMA throughput of the device (TFLOP/s, 2 flops per FMA) from
 * a register-resident FMA kernel: the denominator of the interaction
 * kernels' roofline.  No counterpart in the reference. */
int tg_device_fp32_peak(int device, double *tflops, void *stream);

#ifdef __cplusplus
}
#endif
#endif
