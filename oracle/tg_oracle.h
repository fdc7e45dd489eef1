/*
 * tg_oracle.h -- CPU oracle for the periodic tree-gravity path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: a serial CPU
 * restatement of TigerGrav's gravity evaluation (tree refine, multipoles,
 * dual-list walk, the eight gravity_* kernels, L2L/L2P, kick/drift) plus an
 * FP64 direct Ewald-sum evaluator used as ground truth.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it.
 * The product (tigergrav_b200/libtigergrav_b200.so) never links or calls it.
 *
 * Every function cites the reference file:line it restates.  Positions are the
 * reference's int32 fixed point (x = i * 2^-32 + 0.5, tigergrav/position.hpp:13-37).
 */
#ifndef TG_ORACLE_H
#define TG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tgo_params {
    double theta;    /* opening angle (options::theta, src/options.cpp:54)        */
    double soft_len; /* h (options::soft_len, src/options.cpp:86-88)              */
    double m;        /* particle mass m_tot/problem_size (src/gravity.cpp:186)    */
    double G;        /* gravitational constant (options::G)                        */
    int ewald;       /* periodic Ewald correction on/off (options::ewald)          */
    int leaf_max;    /* parts_per_node (src/options.cpp:52)                        */
} tgo_params;

/* interaction list kinds (CSR per node) */
enum {
    TGO_CC_D = 0, TGO_CP_D = 1, TGO_CC_E = 2, TGO_CP_E = 3, /* node stage  */
    TGO_PC_D = 4, TGO_PP_D = 5, TGO_PC_E = 6, TGO_PP_E = 7, /* leaf stage  */
    TGO_NLIST = 8
};

/* Kernel signatures shared by the restated kernels (tgo_*) and the wrappers
 * around the reference's own kernels (ref_*, oracle/ref_driver.cpp).
 * f is nx x 4 doubles (phi, gx, gy, gz), accumulated with +=.
 * L is 35 doubles (expansion<double>), accumulated with +=.
 * Multipole sources: ym = ny x 17 floats, yx = ny x 3 int32 (multi_src).   */
typedef uint64_t (*tgo_pp_fn)(const tgo_params *, double *f, const int32_t *x, int nx,
                              const int32_t *y, int ny, int do_phi);
typedef uint64_t (*tgo_pc_fn)(const tgo_params *, double *f, const int32_t *x, int nx,
                              const float *ym, const int32_t *yx, int ny);
typedef uint64_t (*tgo_cc_fn)(const tgo_params *, double *L, const int32_t *x,
                              const float *ym, const int32_t *yx, int ny);
typedef uint64_t (*tgo_cp_fn)(const tgo_params *, double *L, const int32_t *x,
                              const int32_t *y, int ny);

/* ---- restated kernels (src/gravity.cpp) ---- */
uint64_t tgo_PP_direct(const tgo_params *, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi);
uint64_t tgo_PC_direct(const tgo_params *, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny);
uint64_t tgo_CC_direct(const tgo_params *, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny);
uint64_t tgo_CP_direct(const tgo_params *, double *L, const int32_t *x, const int32_t *y, int ny);
uint64_t tgo_PP_ewald(const tgo_params *, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi);
uint64_t tgo_PC_ewald(const tgo_params *, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny);
uint64_t tgo_CC_ewald(const tgo_params *, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny);
uint64_t tgo_CP_ewald(const tgo_params *, double *L, const int32_t *x, const int32_t *y, int ny);

/* the same kernels with every interaction computed in double (FP64 oracle) */
uint64_t tgo64_PP_direct(const tgo_params *, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi);
uint64_t tgo64_PC_direct(const tgo_params *, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny);
uint64_t tgo64_CC_direct(const tgo_params *, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny);
uint64_t tgo64_CP_direct(const tgo_params *, double *L, const int32_t *x, const int32_t *y, int ny);
uint64_t tgo64_PP_ewald(const tgo_params *, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi);
uint64_t tgo64_PC_ewald(const tgo_params *, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny);
uint64_t tgo64_CC_ewald(const tgo_params *, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny);
uint64_t tgo64_CP_ewald(const tgo_params *, double *L, const int32_t *x, const int32_t *y, int ny);

/* green_ewald(dX) in the reference's FP32 arithmetic (tigergrav/green.hpp:189-286): D[35] */
void tgo_green_ewald(const float dx[3], float D[35]);
/* green_direct(dX) (tigergrav/green.hpp:167-186): D[35] */
void tgo_green_direct(const float dx[3], float D[35]);
/* L2L: L <<= dX (tigergrav/expansion.hpp:184-233), in double */
void tgo_L2L(double L[35], const double dx[3]);
/* L2P: translate_L2 (tigergrav/expansion.hpp:235-269): out phi, g[3] */
void tgo_L2P(const double L[35], const double dx[3], double out[4]);
/* M2M: M >>= dX (tigergrav/multipole.hpp:116-135), in float */
void tgo_M2M(float M[17], const float dx[3]);

/* ---- solver object (tree + walk + evaluation) ---- */
void *tgo_create(const tgo_params *p);
void tgo_destroy(void *h);
int tgo_set_particles(void *h, const int32_t *x, const float *v, int64_t n);
/* refine restatement (src/tree.cpp:122-201, src/part_vect.cpp:895-933); 0 ok */
int tgo_build(void *h);
/* compute_multipoles restatement (src/tree.cpp:203-296, src/part_vect.cpp:542-635) */
int tgo_multipoles(void *h);
/* kick_fmm list generation (src/tree.cpp:378-635) */
int tgo_walk(void *h);
/* the same lists on nthreads threads (subtrees walked concurrently) */
int tgo_walk_mt(void *h, int nthreads);
/* Evaluate forces along the lists. use_ref: 0 = restated kernels (reference
 * arithmetic), 1 = the reference's kernels loaded by tgo_load_reference,
 * 2 = restated kernels in FP64.  nthreads >= 1.
 * leaf_subset (may be NULL): evaluate only these leaves (node ids) and the
 * nodes on their root paths; forces of other particles are left at zero.   */
int tgo_evaluate(void *h, int use_ref, int nthreads, const int32_t *leaf_subset, int64_t nsubset);
int tgo_load_reference(void *h, const char *so_path);

int64_t tgo_num_nodes(void *h);
int64_t tgo_num_particles(void *h);
/* node arrays, each of length num_nodes (NULL to skip):
 *   boxid (u64, 1<<level | prefix), level, pbegin, pend, child0 (-1 leaf),
 *   parent (-1 root), x (3 int32), r (float), rmax (float), m (17 floats)    */
int tgo_get_nodes(void *h, uint64_t *boxid, int32_t *level, int64_t *pbegin, int64_t *pend,
                  int32_t *child0, int32_t *parent, int32_t *x, float *r, float *rmax, float *m);
/* particle order after the partition: perm[i] = caller index of sorted particle i */
int tgo_get_perm(void *h, int64_t *perm);
/* CSR list of kind k: offsets (num_nodes+1), ids (offsets[num_nodes]) */
int64_t tgo_list_size(void *h, int kind);
int tgo_get_list(void *h, int kind, int64_t *offsets, int32_t *ids);
/* forces in caller order: phi[n], g[n*3] */
int tgo_get_forces(void *h, double *phi, double *g);
/* per-node expansions (num_nodes x 35), after tgo_evaluate */
int tgo_get_expansions(void *h, double *L);
/* statistics: interaction_stats as the reference files them (tigergrav/tree.hpp:84-114)
 * [PP_d, PP_e, CC_d, CC_e, CP_d, CP_e] plus clean counts
 * [pairs PP_d, PP_e, PC_d, PC_e, CC_d, CC_e, CP_d, CP_e] and flops (reference convention) */
int tgo_get_stats(void *h, uint64_t ref_stats[6], uint64_t counts[8], uint64_t *flops);
/* host throughput of each interaction kind (ns per interaction, list-kind
 * order), sampled over random sinks for at most budget_s seconds per kind */
int tgo_kind_costs(void *h, int use_ref, int nthreads, double budget_s, uint64_t seed, double *ns_per, uint64_t *done);

/* kick/drift (clean KDK restatement of src/part_vect.cpp:341-436, 493-540) */
int tgo_kick(void *h, double dt);                 /* v += g * G * dt  (float v, double math) */
int tgo_drift(void *h, double dt, double *ekin);  /* x = wrap(x + v dt), requantised */
int tgo_get_particles(void *h, int32_t *x, float *v); /* caller order */
/* energy / momentum reductions in double: out[0]=ekin, [1]=epot, [2..4]=sum v/N */
int tgo_energy(void *h, double out[5]);

/* ---- FP64 direct Ewald-sum ground truth ----
 * For each sample particle, the full periodic force and potential from all n
 * particles (mass m), nearest-image GADGET spline softening inside h, computed
 * with an independent Ewald split (parameter alpha) in double precision.       */
int tgo_truth(const int32_t *x, int64_t n, const int64_t *samples, int64_t ns,
              double m, double h, double alpha, int nthreads, double *phi, double *g);
/* The reference-convention periodic correction (alpha=2, 305 real + 123 Fourier
 * vectors, tigergrav/green.hpp:8-59,189-286) evaluated in double: out[0]=phi, [1..3]=g */
void tgo_ewald_corr_f64(const double dx[3], double out[4]);

#ifdef __cplusplus
}
#endif
#endif
