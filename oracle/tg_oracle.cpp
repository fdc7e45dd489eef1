/*
 * tg_oracle.cpp -- serial CPU restatement of TigerGrav's periodic gravity
 * evaluation.  TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Arithmetic follows the reference source as written under ISO C++ rules
 * (built with -ffp-contract=off): FP32 per interaction, FP64 accumulation,
 * FP64 for positions / centres of mass / opening criteria.  Where the
 * reference relies on approximations (A&S 7.1.26 erfc, polynomial exp and a
 * Chebyshev sine, tigergrav/simd.hpp:556-692) this file uses A&S 7.1.26 with
 * libm expf and libm sinf/cosf; those differ from the reference's by ~1e-7.
 */
#include "tg_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <thread>
#include <chrono>
#include <vector>

namespace {

constexpr double POS_MAX = 4294967296.0;
constexpr double POS_INV = 1.0 / POS_MAX;
constexpr int MP = 17;
constexpr int LP = 35;

/* tigergrav/position.hpp:18-37 */
inline double pos_to_double(int32_t x) { return ((double)x) * POS_INV + 0.5; }
inline int32_t double_to_pos(double x) {
    const double y = x - 0.5;
    long z = std::lround(y * POS_MAX);
    if (z >= POS_MAX / 2.0) {
        z -= (long)POS_MAX;
    }
    return (int32_t)(uint32_t)(uint64_t)z;
}

/* ---- symmetric-tensor storage (tigergrav/multipole.hpp:58-82, expansion.hpp:77-137):
 * slots of each order enumerate the sorted index tuples lexicographically. */
struct SymIdx {
    int t2[3][3];
    int t3[3][3][3];
    int t4[3][3][3][3];
    SymIdx() {
        int k = 0;
        for (int a = 0; a < 3; a++)
            for (int b = a; b < 3; b++) {
                t2[a][b] = t2[b][a] = k++;
            }
        k = 0;
        for (int a = 0; a < 3; a++)
            for (int b = a; b < 3; b++)
                for (int c = b; c < 3; c++) {
                    int p[3] = {a, b, c};
                    do {
                        t3[p[0]][p[1]][p[2]] = k;
                    } while (std::next_permutation(p, p + 3));
                    k++;
                }
        k = 0;
        for (int a = 0; a < 3; a++)
            for (int b = a; b < 3; b++)
                for (int c = b; c < 3; c++)
                    for (int d = c; d < 3; d++) {
                        int p[4] = {a, b, c, d};
                        do {
                            t4[p[0]][p[1]][p[2]][p[3]] = k;
                        } while (std::next_permutation(p, p + 4));
                        k++;
                    }
    }
};
const SymIdx SI;

inline int E0() { return 0; }
inline int E1(int a) { return 1 + a; }
inline int E2(int a, int b) { return 4 + SI.t2[a][b]; }
inline int E3(int a, int b, int c) { return 10 + SI.t3[a][b][c]; }
inline int E4(int a, int b, int c, int d) { return 20 + SI.t4[a][b][c][d]; }
inline int M2i(int a, int b) { return 1 + SI.t2[a][b]; }
inline int M3i(int a, int b, int c) { return 7 + SI.t3[a][b][c]; }

/* expansion_factors (tigergrav/expansion.hpp:162-182), accumulated in T */
template <class T>
struct Factors {
    T f[LP];
    Factors() {
        for (int i = 0; i < LP; i++) f[i] = T(0.0);
        f[E0()] += T(1);
        for (int a = 0; a < 3; ++a) {
            f[E1(a)] += T(1.0);
            for (int b = 0; b < 3; ++b) {
                f[E2(a, b)] += T(0.5);
                for (int c = 0; c < 3; ++c) {
                    f[E3(a, b, c)] += T(1.0 / 6.0);
                    for (int d = 0; d < 3; ++d) {
                        f[E4(a, b, c, d)] += T(1.0 / 24.0);
                    }
                }
            }
        }
    }
};
const Factors<float> FF;
const Factors<double> FD;

/* ---- Ewald lattice tables (tigergrav/green.hpp:8-59) ---- */
struct EwaldIdx {
    std::vector<std::array<float, 3>> v;
    explicit EwaldIdx(int n2max) {
        const int nmax = (int)std::sqrt((float)n2max) + 1;
        for (int i = -nmax; i <= nmax; i++)
            for (int j = -nmax; j <= nmax; j++)
                for (int k = -nmax; k <= nmax; k++)
                    if (i * i + j * j + k * k <= n2max) v.push_back({(float)i, (float)j, (float)k});
        std::stable_sort(v.begin(), v.end(), [](const std::array<float, 3> &a, const std::array<float, 3> &b) {
            return a[0] * a[0] + a[1] * a[1] + a[2] * a[2] > b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
        });
    }
};
const EwaldIdx REAL_IDX(17);
const EwaldIdx FOUR_IDX(9);

struct PeriodicParts {
    std::vector<std::array<float, LP>> H;
    PeriodicParts() {
        for (auto &hv : FOUR_IDX.v) {
            const float h[3] = {hv[0], hv[1], hv[2]};
            const float h2 = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
            std::array<float, LP> D;
            D.fill(0.0f);
            if (h2 > 0) {
                const float c0 = 1.0 / h2 * std::exp(-M_PI * M_PI * h2 / 4.0);
                D[E0()] = -(1.0 / M_PI) * c0;
                for (int a = 0; a < 3; a++) {
                    D[E1(a)] = 2.0 * h[a] * c0;
                    for (int b = 0; b <= a; b++) {
                        D[E2(a, b)] = 4.0 * M_PI * h[a] * h[b] * c0;
                        for (int c = 0; c <= b; c++) {
                            D[E3(a, b, c)] = -8.0 * M_PI * M_PI * h[a] * h[b] * h[c] * c0;
                            for (int d = 0; d <= c; d++) {
                                D[E4(a, b, c, d)] = -16.0 * M_PI * M_PI * M_PI * h[a] * h[b] * h[c] * h[d] * c0;
                            }
                        }
                    }
                }
            }
            H.push_back(D);
        }
    }
};
const PeriodicParts PERIODIC;

template <class R> struct Fac;
template <> struct Fac<float> {
    static const Factors<float> &get() { return FF; }
};
template <> struct Fac<double> {
    static const Factors<double> &get() { return FD; }
};

/* periodic_parts without the float rounding of c0, for the FP64 kernels */
struct PeriodicPartsD {
    std::vector<std::array<double, LP>> H;
    PeriodicPartsD() {
        for (auto &hv : FOUR_IDX.v) {
            const double h[3] = {hv[0], hv[1], hv[2]};
            const double h2 = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
            std::array<double, LP> D;
            D.fill(0.0);
            if (h2 > 0) {
                const double c0 = 1.0 / h2 * std::exp(-M_PI * M_PI * h2 / 4.0);
                D[E0()] = -(1.0 / M_PI) * c0;
                for (int a = 0; a < 3; a++) {
                    D[E1(a)] = 2.0 * h[a] * c0;
                    for (int b = 0; b <= a; b++) {
                        D[E2(a, b)] = 4.0 * M_PI * h[a] * h[b] * c0;
                        for (int c = 0; c <= b; c++) {
                            D[E3(a, b, c)] = -8.0 * M_PI * M_PI * h[a] * h[b] * h[c] * c0;
                            for (int d = 0; d <= c; d++)
                                D[E4(a, b, c, d)] = -16.0 * M_PI * M_PI * M_PI * h[a] * h[b] * h[c] * h[d] * c0;
                        }
                    }
                }
            }
            H.push_back(D);
        }
    }
};
const PeriodicPartsD PERIODIC_D;
template <class R> struct Per;
template <> struct Per<float> {
    static const PeriodicParts &get() { return PERIODIC; }
};
template <> struct Per<double> {
    static const PeriodicPartsD &get() { return PERIODIC_D; }
};
template <class R> inline void load_m(R *M, const float *ym) {
    for (int k = 0; k < MP; k++) M[k] = (R)ym[k];
}

/* The kernels in the reference's arithmetic (R = float) and in plain FP64
 * (R = double, the double-precision oracle for the FP64 GPU path). */
namespace k32 {
using R = float;
#include "tg_oracle_kernels.inc"
} // namespace k32
namespace k64 {
using R = double;
#include "tg_oracle_kernels.inc"
} // namespace k64

} // namespace

extern "C" {

uint64_t tgo_PP_direct(const tgo_params *p, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi) {
    return k32::k_PP_direct(p, f, x, nx, y, ny, do_phi);
}
uint64_t tgo_PC_direct(const tgo_params *p, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny) {
    return k32::k_PC_direct(p, f, x, nx, ym, yx, ny);
}
uint64_t tgo_CC_direct(const tgo_params *p, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny) {
    return k32::k_CC_direct(p, L, x, ym, yx, ny);
}
uint64_t tgo_CP_direct(const tgo_params *p, double *L, const int32_t *x, const int32_t *y, int ny) {
    return k32::k_CP_direct(p, L, x, y, ny);
}
uint64_t tgo_PP_ewald(const tgo_params *p, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi) {
    return k32::k_PP_ewald(p, f, x, nx, y, ny, do_phi);
}
uint64_t tgo_PC_ewald(const tgo_params *p, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny) {
    return k32::k_PC_ewald(p, f, x, nx, ym, yx, ny);
}
uint64_t tgo_CC_ewald(const tgo_params *p, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny) {
    return k32::k_CC_ewald(p, L, x, ym, yx, ny);
}
uint64_t tgo_CP_ewald(const tgo_params *p, double *L, const int32_t *x, const int32_t *y, int ny) {
    return k32::k_CP_ewald(p, L, x, y, ny);
}
uint64_t tgo64_PP_direct(const tgo_params *p, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi) {
    return k64::k_PP_direct(p, f, x, nx, y, ny, do_phi);
}
uint64_t tgo64_PC_direct(const tgo_params *p, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny) {
    return k64::k_PC_direct(p, f, x, nx, ym, yx, ny);
}
uint64_t tgo64_CC_direct(const tgo_params *p, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny) {
    return k64::k_CC_direct(p, L, x, ym, yx, ny);
}
uint64_t tgo64_CP_direct(const tgo_params *p, double *L, const int32_t *x, const int32_t *y, int ny) {
    return k64::k_CP_direct(p, L, x, y, ny);
}
uint64_t tgo64_PP_ewald(const tgo_params *p, double *f, const int32_t *x, int nx, const int32_t *y, int ny, int do_phi) {
    return k64::k_PP_ewald(p, f, x, nx, y, ny, do_phi);
}
uint64_t tgo64_PC_ewald(const tgo_params *p, double *f, const int32_t *x, int nx, const float *ym, const int32_t *yx, int ny) {
    return k64::k_PC_ewald(p, f, x, nx, ym, yx, ny);
}
uint64_t tgo64_CC_ewald(const tgo_params *p, double *L, const int32_t *x, const float *ym, const int32_t *yx, int ny) {
    return k64::k_CC_ewald(p, L, x, ym, yx, ny);
}
uint64_t tgo64_CP_ewald(const tgo_params *p, double *L, const int32_t *x, const int32_t *y, int ny) {
    return k64::k_CP_ewald(p, L, x, y, ny);
}

void tgo_green_ewald(const float dx[3], float D[35]) { k32::green_ewald(dx, D); }
void tgo_green_direct(const float dx[3], float D[35]) { k32::green_direct(dx, D); }

/* expansion<double>::operator<<= (tigergrav/expansion.hpp:184-233) */
void tgo_L2L(double *me, const double *dX) {
    const auto &factor = FD.f;
    for (int a = 0; a < 3; a++) {
        me[E0()] += me[E1(a)] * dX[a];
        for (int b = 0; b <= a; b++) {
            me[E0()] += me[E2(a, b)] * dX[a] * dX[b] * factor[E2(a, b)];
            for (int c = 0; c <= b; c++) {
                me[E0()] += me[E3(a, b, c)] * dX[a] * dX[b] * dX[c] * factor[E3(a, b, c)];
                for (int d = 0; d <= c; d++) {
                    me[E0()] += me[E4(a, b, c, d)] * dX[a] * dX[b] * dX[c] * dX[d] * factor[E4(a, b, c, d)];
                }
            }
        }
    }
    for (int a = 0; a < 3; a++) {
        for (int b = 0; b < 3; b++) {
            me[E1(a)] += me[E2(a, b)] * dX[b];
            for (int c = 0; c <= b; c++) {
                me[E1(a)] += me[E3(a, b, c)] * dX[b] * dX[c] * factor[E2(b, c)];
                for (int d = 0; d <= c; d++) {
                    me[E1(a)] += me[E4(a, b, c, d)] * dX[b] * dX[c] * dX[d] * factor[E3(b, c, d)];
                }
            }
        }
    }
    for (int a = 0; a < 3; a++) {
        for (int b = 0; b <= a; b++) {
            for (int c = 0; c < 3; c++) {
                me[E2(a, b)] += me[E3(a, b, c)] * dX[c];
                for (int d = 0; d <= c; d++) {
                    me[E2(a, b)] += me[E4(a, b, c, d)] * dX[c] * dX[d] * factor[E2(c, d)];
                }
            }
        }
    }
    for (int a = 0; a < 3; a++)
        for (int b = 0; b <= a; b++)
            for (int c = 0; c <= b; c++)
                for (int d = 0; d < 3; d++) me[E3(a, b, c)] += me[E4(a, b, c, d)] * dX[d];
}

/* expansion<double>::translate_L2 (tigergrav/expansion.hpp:235-269) */
void tgo_L2P(const double *me, const double *dX, double *out) {
    const auto &factor = FD.f;
    double phi = me[E0()];
    for (int a = 0; a < 3; a++) {
        phi += me[E1(a)] * dX[a];
        for (int b = a; b < 3; b++) {
            phi += me[E2(a, b)] * dX[a] * dX[b] * factor[E2(a, b)];
            for (int c = b; c < 3; c++) {
                phi += me[E3(a, b, c)] * dX[a] * dX[b] * dX[c] * factor[E3(a, b, c)];
                for (int d = c; d < 3; d++) {
                    phi += me[E4(a, b, c, d)] * dX[a] * dX[b] * dX[c] * dX[d] * factor[E4(a, b, c, d)];
                }
            }
        }
    }
    out[0] = phi;
    for (int a = 0; a < 3; a++) {
        double g = -me[E1(a)];
        for (int b = 0; b < 3; b++) {
            g -= me[E2(a, b)] * dX[b];
            for (int c = b; c < 3; c++) {
                g -= me[E3(a, b, c)] * dX[b] * dX[c] * factor[E2(b, c)];
                for (int d = c; d < 3; d++) {
                    g -= me[E4(a, b, c, d)] * dX[b] * dX[c] * dX[d] * factor[E3(b, c, d)];
                }
            }
        }
        out[1 + a] = g;
    }
}

/* multipole<float>::operator>>= (tigergrav/multipole.hpp:116-135) */
void tgo_M2M(float *me, const float *Y) {
    for (int p = 0; p < 3; p++)
        for (int q = p; q < 3; q++)
            for (int l = q; l < 3; l++) {
                float &m3 = me[M3i(p, q, l)];
                m3 += me[0] * Y[p] * Y[q] * Y[l];
                m3 += me[M2i(p, q)] * Y[l];
                m3 += me[M2i(q, l)] * Y[p];
                m3 += me[M2i(l, p)] * Y[q];
            }
    for (int p = 0; p < 3; p++)
        for (int q = p; q < 3; q++) me[M2i(p, q)] += me[0] * Y[p] * Y[q];
}

} // extern "C"

/* ======================= solver object ======================= */
namespace {

struct Node {
    uint64_t boxid = 1;
    int level = 0;
    int64_t pb = 0, pe = 0;
    int32_t child0 = -1, parent = -1;
    float m[MP];
    float r = 0.0f;
    int32_t x[3] = {0, 0, 0};
    uint64_t num_active = 0;
    double prmin[3], prmax[3]; /* rc.r of compute_multipoles */
    double amin[3], amax[3];   /* particle AABB (part_vect_range) */
    float rmax = 0.0f;         /* range_max_span of the particle AABB (tree.cpp:406) */
    uint64_t N = 0;
    bool leaf() const { return child0 < 0; }
};

struct CheckItem {
    int32_t node;
    bool opened;
};

typedef void (*ref_init_fn)(double theta, double soft_len, double m_tot, uint64_t n, int ewald, double G);

struct Solver {
    tgo_params p;
    int64_t n = 0;
    std::vector<int32_t> x;   /* sorted order, 3 per particle */
    std::vector<float> v;     /* sorted order */
    std::vector<int64_t> perm;/* sorted index -> caller index */
    std::vector<Node> nodes;
    std::vector<std::vector<int32_t>> lists[TGO_NLIST];
    std::vector<double> f;    /* sorted order, 4 per particle */
    std::vector<double> L;    /* per node, 35 */
    uint64_t ref_stats[6] = {0};
    uint64_t counts[8] = {0};
    std::atomic<uint64_t> flops{0};
    uint64_t p2m_flops = 0; /* compute_multipoles share, src/tree.cpp:234 */
    double theta_inv = 0;
    float r_ewald = 0;
    /* reference kernel table */
    void *dl = nullptr;
    tgo_pp_fn ref_pp_d = nullptr, ref_pp_e = nullptr;
    tgo_pc_fn ref_pc_d = nullptr, ref_pc_e = nullptr;
    tgo_cc_fn ref_cc_d = nullptr, ref_cc_e = nullptr;
    tgo_cp_fn ref_cp_d = nullptr, ref_cp_e = nullptr;
};

/* box_id_to_range (src/range.cpp:134-168) */
void box_id_to_range(uint64_t id, double *mn, double *mx) {
    double x[3] = {0.0, 0.0, 0.0}, dx[3] = {1.0, 1.0, 1.0};
    while (id != 1) {
        const double tmp1 = x[0], tmp2 = dx[0];
        x[0] = x[2];
        x[2] = x[1];
        x[1] = tmp1;
        dx[0] = dx[2];
        dx[2] = dx[1];
        dx[1] = tmp2;
        if (id & 1) {
            x[0] = 0.5 * x[0] + 0.5;
        } else {
            x[0] = 0.5 * x[0];
        }
        dx[0] *= 0.5;
        id >>= 1;
    }
    for (int d = 0; d < 3; d++) {
        mn[d] = x[d];
        mx[d] = x[d] + dx[d];
    }
}

/* part_vect_sort (src/part_vect.cpp:895-933): swap partition, returns split */
int64_t partition(Solver &S, int64_t b, int64_t e, double xmid, int dim) {
    if (e == b) return e;
    int64_t lo = b, hi = e;
    auto swap_parts = [&](int64_t i, int64_t j) {
        for (int d = 0; d < 3; d++) std::swap(S.x[3 * i + d], S.x[3 * j + d]);
        for (int d = 0; d < 3; d++) std::swap(S.v[3 * i + d], S.v[3 * j + d]);
        std::swap(S.perm[i], S.perm[j]);
    };
    while (lo < hi) {
        if (pos_to_double(S.x[3 * lo + dim]) >= xmid) {
            while (lo != hi) {
                hi--;
                if (pos_to_double(S.x[3 * hi + dim]) < xmid) {
                    swap_parts(lo, hi);
                    break;
                }
            }
        }
        lo++;
    }
    return hi;
}

inline double vabs(const double *a) {
    double r = a[0] * a[0];
    r += a[1] * a[1];
    r += a[2] * a[2];
    return std::sqrt(r);
}

/* ewald_near_separation (src/gravity.cpp:10-18) */
inline double near_sep(const double *x) {
    double d = 0.0;
    for (int dim = 0; dim < 3; dim++) {
        const double absx = std::abs(x[dim]);
        const double this_d = std::min(absx, (double)1.0 - absx);
        d += this_d * this_d;
    }
    return std::sqrt(d);
}

/* interaction_stats of one walk (or of one thread's share of it) */
struct Tally {
    uint64_t ref_stats[6] = {0, 0, 0, 0, 0, 0};
    uint64_t counts[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    void add(const Tally &o) {
        for (int k = 0; k < 6; k++) ref_stats[k] += o.ref_stats[k];
        for (int k = 0; k < 8; k++) counts[k] += o.counts[k];
    }
};
/* a node with the check lists its parent handed down */
struct WalkTask {
    int32_t node;
    std::vector<CheckItem> d, e;
};

void walk_node(Solver &S, int32_t n, std::vector<CheckItem> dlist, std::vector<CheckItem> elist, Tally &T,
               std::vector<WalkTask> *defer);

} // namespace

extern "C" {

void *tgo_create(const tgo_params *p) {
    Solver *S = new Solver();
    S->p = *p;
    S->theta_inv = 1.0 / p->theta;
    S->r_ewald = (float)(2.0 * p->theta * std::pow(1.0e-3 / 8.0, 1.0 / 3.0));
    return S;
}

void tgo_destroy(void *h) {
    Solver *S = (Solver *)h;
    if (S->dl) dlclose(S->dl);
    delete S;
}

int tgo_set_particles(void *h, const int32_t *x, const float *v, int64_t n) {
    Solver &S = *(Solver *)h;
    if (n < 1) return -1;
    S.n = n;
    S.x.assign(x, x + 3 * n);
    if (v) S.v.assign(v, v + 3 * n);
    else S.v.assign(3 * n, 0.0f);
    S.perm.resize(n);
    for (int64_t i = 0; i < n; i++) S.perm[i] = i;
    S.nodes.clear();
    return 0;
}

/* refine (src/tree.cpp:122-201), breadth first: node ids are level order,
 * increasing box id within a level.  The depth is capped at 63 levels (box
 * ids fit 64 bits); a node that would need level 64 is an error (-2). */
int tgo_build(void *h) {
    Solver &S = *(Solver *)h;
    S.nodes.clear();
    Node root;
    root.boxid = 1;
    root.level = 0;
    root.pb = 0;
    root.pe = S.n;
    S.nodes.push_back(root);
    size_t lvl_begin = 0, lvl_end = 1;
    while (lvl_begin < lvl_end) {
        for (size_t i = lvl_begin; i < lvl_end; i++) {
            Node nd = S.nodes[i];
            if (nd.pe - nd.pb > S.p.leaf_max) {
                if (nd.level >= 63) return -2;
                double mn[3], mx[3];
                box_id_to_range(nd.boxid, mn, mx);
                double max_span = 0.0;
                int max_dim = 0;
                for (int dim = 0; dim < 3; dim++) {
                    const double span = mx[dim] - mn[dim];
                    if (span > max_span) {
                        max_span = span;
                        max_dim = dim;
                    }
                }
                const double mid = (mx[max_dim] + mn[max_dim]) * 0.5;
                const int64_t split = partition(S, nd.pb, nd.pe, mid, max_dim);
                Node c0, c1;
                c0.boxid = nd.boxid << 1;
                c1.boxid = (nd.boxid << 1) + 1;
                c0.level = c1.level = nd.level + 1;
                c0.pb = nd.pb;
                c0.pe = split;
                c1.pb = split;
                c1.pe = nd.pe;
                c0.parent = c1.parent = (int32_t)i;
                S.nodes[i].child0 = (int32_t)S.nodes.size();
                S.nodes.push_back(c0);
                S.nodes.push_back(c1);
            }
        }
        lvl_begin = lvl_end;
        lvl_end = S.nodes.size();
    }
    return 0;
}

/* compute_multipoles (src/tree.cpp:203-296) with part_vect_center_of_mass,
 * part_vect_multipole_info and part_vect_range (src/part_vect.cpp:542-635,
 * 935-968).  Children are processed before parents (reverse level order). */
int tgo_multipoles(void *h) {
    Solver &S = *(Solver *)h;
    const float mass = (float)S.p.m;
    S.p2m_flops = 0;
    for (int64_t i = (int64_t)S.nodes.size() - 1; i >= 0; i--) {
        Node &nd = S.nodes[i];
        const int64_t cnt = nd.pe - nd.pb;
        if (cnt == 0) {
            double mn[3], mx[3];
            box_id_to_range(nd.boxid, mn, mx);
            nd.N = 0;
            for (int k = 0; k < MP; k++) nd.m[k] = 0.0f;
            for (int d = 0; d < 3; d++) nd.x[d] = double_to_pos(0.5 * (mx[d] - mn[d]));
            nd.num_active = 0;
            nd.r = 0.0f;
            for (int d = 0; d < 3; d++) {
                nd.prmin[d] = mn[d];
                nd.prmax[d] = mx[d];
            }
            continue;
        }
        /* particle AABB, part_vect_range */
        for (int d = 0; d < 3; d++) {
            nd.amax[d] = 0.0;
            nd.amin[d] = 1.0;
        }
        for (int64_t k = nd.pb; k < nd.pe; k++)
            for (int d = 0; d < 3; d++) {
                const double xx = pos_to_double(S.x[3 * k + d]);
                nd.amax[d] = std::max(nd.amax[d], xx);
                nd.amin[d] = std::min(nd.amin[d], xx);
            }
        {
            double s = 0.0;
            for (int d = 0; d < 3; d++) s += std::pow(nd.amax[d] - nd.amin[d], 2);
            nd.rmax = (float)std::sqrt(s);
        }
        if (nd.leaf()) {
            double com[3] = {0, 0, 0};
            for (int64_t k = nd.pb; k < nd.pe; k++)
                for (int d = 0; d < 3; d++) com[d] += pos_to_double(S.x[3 * k + d]);
            for (int d = 0; d < 3; d++) com[d] = com[d] / double(cnt);
            nd.N = cnt;
            for (int d = 0; d < 3; d++) nd.x[d] = double_to_pos(com[d]);
            const double Xcom[3] = {pos_to_double(nd.x[0]), pos_to_double(nd.x[1]), pos_to_double(nd.x[2])};
            /* 16 lanes: particle k goes to lane (k - pb) % 16, lanes summed in order */
            float lane[16][MP];
            for (int l = 0; l < 16; l++)
                for (int k = 0; k < MP; k++) lane[l][k] = 0.0f;
            for (int64_t k = nd.pb; k < nd.pe; k++) {
                float *M = lane[(k - nd.pb) % 16];
                float dx[3];
                for (int d = 0; d < 3; d++) dx[d] = (float)(pos_to_double(S.x[3 * k + d]) - Xcom[d]);
                M[0] += mass;
                for (int j = 0; j < 3; j++)
                    for (int q = 0; q <= j; q++) {
                        const float Xjk = dx[j] * dx[q];
                        M[M2i(j, q)] += mass * Xjk;
                        for (int l = 0; l <= q; l++) M[M3i(j, q, l)] += mass * Xjk * dx[l];
                    }
            }
            for (int k = 0; k < MP; k++) {
                float sum = 0.0f;
                for (int l = 0; l < 16; l++) sum += lane[l][k];
                nd.m[k] = sum;
            }
            nd.r = 0.0f;
            nd.num_active = 0;
            for (int64_t k = nd.pb; k < nd.pe; k++) {
                double dd[3];
                for (int d = 0; d < 3; d++) dd[d] = pos_to_double(S.x[3 * k + d]) - Xcom[d];
                nd.r = std::max(nd.r, (float)vabs(dd));
                nd.num_active++;
            }
            for (int d = 0; d < 3; d++) {
                nd.prmin[d] = nd.amin[d];
                nd.prmax[d] = nd.amax[d];
            }
            S.p2m_flops += (uint64_t)cnt * 64;
        } else {
            const Node &ml = S.nodes[nd.child0];
            const Node &mr = S.nodes[nd.child0 + 1];
            nd.N = ml.N + mr.N;
            double xs[3];
            for (int d = 0; d < 3; d++)
                xs[d] = (pos_to_double(ml.x[d]) * (double)ml.N + pos_to_double(mr.x[d]) * (double)mr.N) / (double)nd.N;
            for (int d = 0; d < 3; d++) nd.x[d] = double_to_pos(xs[d]);
            double X[3], XL[3], XR[3];
            for (int d = 0; d < 3; d++) {
                X[d] = pos_to_double(nd.x[d]);
                XL[d] = pos_to_double(ml.x[d]);
                XR[d] = pos_to_double(mr.x[d]);
            }
            float ML[MP], MR[MP];
            std::memcpy(ML, ml.m, sizeof(ML));
            std::memcpy(MR, mr.m, sizeof(MR));
            float dl[3], dr[3];
            for (int d = 0; d < 3; d++) {
                dl[d] = (float)(XL[d] - X[d]);
                dr[d] = (float)(XR[d] - X[d]);
            }
            tgo_M2M(ML, dl);
            tgo_M2M(MR, dr);
            for (int k = 0; k < MP; k++) nd.m[k] = ML[k] + MR[k];
            nd.num_active = ml.num_active + mr.num_active;
            double dld[3], drd[3];
            for (int d = 0; d < 3; d++) {
                dld[d] = XL[d] - X[d];
                drd[d] = XR[d] - X[d];
            }
            if (ml.N == 0) {
                nd.r = mr.r;
            } else if (mr.N == 0) {
                nd.r = ml.r;
            } else {
                nd.r = (float)std::max(vabs(dld) + ml.r, vabs(drd) + mr.r);
            }
            for (int d = 0; d < 3; d++) {
                nd.prmax[d] = std::max(ml.prmax[d], mr.prmax[d]);
                nd.prmin[d] = std::min(ml.prmin[d], mr.prmin[d]);
            }
            double rmax = 0.0;
            for (int c = 0; c < 8; c++) {
                double dd[3];
                for (int d = 0; d < 3; d++) dd[d] = X[d] - (((c >> d) & 1) ? nd.prmax[d] : nd.prmin[d]);
                rmax = std::max(rmax, vabs(dd));
            }
            nd.r = std::min(nd.r, (float)rmax);
        }
    }
    return 0;
}

int tgo_walk(void *h) {
    Solver &S = *(Solver *)h;
    for (int k = 0; k < TGO_NLIST; k++) {
        S.lists[k].assign(S.nodes.size(), std::vector<int32_t>());
    }
    std::vector<CheckItem> root = {{0, false}};
    Tally T;
    walk_node(S, 0, root, root, T, nullptr);
    for (int k = 0; k < 6; k++) S.ref_stats[k] = T.ref_stats[k];
    for (int k = 0; k < 8; k++) S.counts[k] = T.counts[k];
    return 0;
}

} // extern "C"

namespace {

/* kick_fmm list generation (src/tree.cpp:378-635).  The per-node criterion
 * keeps the reference's mixed float/double arithmetic: (r_a + r_b) is a
 * float sum, theta_inv and h are doubles. */
void walk_node(Solver &S, int32_t n, std::vector<CheckItem> dchecklist, std::vector<CheckItem> echecklist, Tally &T,
               std::vector<WalkTask> *defer) {
    const Node &nd = S.nodes[n];
    if (nd.pe - nd.pb == 0) return;
    const double h = S.p.soft_len;
    const double X[3] = {pos_to_double(nd.x[0]), pos_to_double(nd.x[1]), pos_to_double(nd.x[2])};
    const float rmax = nd.rmax;
    const bool ewald = S.p.ewald != 0;
    auto dsep = [&](const Node &c) {
        double dX[3];
        for (int d = 0; d < 3; d++) dX[d] = X[d] - pos_to_double(c.x[d]);
        return ewald ? near_sep(dX) : vabs(dX);
    };
    auto efar = [&](const Node &c) {
        double dX[3];
        for (int d = 0; d < 3; d++) dX[d] = X[d] - pos_to_double(c.x[d]);
        const double dx = std::max(0.25, near_sep(dX));
        double dot = dX[0] * dX[0];
        dot += dX[1] * dX[1];
        dot += dX[2] * dX[2];
        if (dot > 0.0) {
            return dx > (double)(nd.r + c.r) * S.theta_inv && dx > (double)(nd.r + c.r) + h;
        } else {
            return rmax < S.r_ewald;
        }
    };
    std::vector<CheckItem> next_d, next_e;
    std::vector<int32_t> dfuts, efuts;
    uint64_t dsource_count = 0, esource_count = 0;
    for (auto c : dchecklist) {
        const Node &C = S.nodes[c.node];
        if (C.pe == C.pb) continue;
        const double dx = dsep(C);
        const bool far = dx > (double)(nd.r + C.r) * S.theta_inv && dx > (double)(nd.r + C.r) + h;
        if (far) {
            if (c.opened) {
                S.lists[TGO_CP_D][n].push_back(c.node);
                dsource_count += C.pe - C.pb;
            } else {
                S.lists[TGO_CC_D][n].push_back(c.node);
            }
        } else {
            if (C.leaf()) {
                c.opened = true;
                next_d.push_back(c);
            } else {
                dfuts.push_back(c.node);
            }
        }
    }
    if (ewald) {
        for (auto c : echecklist) {
            const Node &C = S.nodes[c.node];
            if (C.pe == C.pb) continue;
            const bool far = efar(C);
            if (far) {
                if (c.opened) {
                    S.lists[TGO_CP_E][n].push_back(c.node);
                    esource_count += C.pe - C.pb;
                } else {
                    S.lists[TGO_CC_E][n].push_back(c.node);
                }
            } else {
                if (C.leaf()) {
                    c.opened = true;
                    next_e.push_back(c);
                } else {
                    efuts.push_back(c.node);
                }
            }
        }
    }
    T.ref_stats[2] += S.lists[TGO_CC_D][n].size();
    T.ref_stats[4] += dsource_count;
    T.counts[4] += S.lists[TGO_CC_D][n].size();
    T.counts[6] += dsource_count;
    if (ewald) {
        T.ref_stats[3] += S.lists[TGO_CC_E][n].size();
        T.ref_stats[5] += esource_count;
        T.counts[5] += S.lists[TGO_CC_E][n].size();
        T.counts[7] += esource_count;
    }
    for (auto f : dfuts) {
        const int32_t c0 = S.nodes[f].child0;
        next_d.push_back({c0, false});
        next_d.push_back({c0 + 1, false});
    }
    for (auto f : efuts) {
        const int32_t c0 = S.nodes[f].child0;
        next_e.push_back({c0, false});
        next_e.push_back({c0 + 1, false});
    }
    if (!nd.leaf()) {
        if (defer) { /* the children become tasks of a parallel walk */
            defer->push_back({nd.child0, next_d, next_e});
            defer->push_back({nd.child0 + 1, std::move(next_d), std::move(next_e)});
            return;
        }
        walk_node(S, nd.child0, next_d, next_e, T, nullptr);
        walk_node(S, nd.child0 + 1, next_d, next_e, T, nullptr);
        return;
    }
    /* leaf drain (src/tree.cpp:530-602) */
    const uint64_t nsink = nd.pe - nd.pb;
    dchecklist.swap(next_d);
    next_d.clear();
    dsource_count = 0;
    while (!dchecklist.empty()) {
        dfuts.clear();
        for (auto c : dchecklist) {
            const Node &C = S.nodes[c.node];
            if (C.pe == C.pb) continue;
            const double dx = dsep(C);
            const bool far = dx > (double)(nd.r + C.r) * S.theta_inv && dx > (double)(nd.r + C.r) + h;
            if (c.opened) {
                S.lists[TGO_PP_D][n].push_back(c.node);
                dsource_count += C.pe - C.pb;
            } else if (far) {
                S.lists[TGO_PC_D][n].push_back(c.node);
            } else if (C.leaf()) {
                c.opened = true;
                next_d.push_back(c);
            } else {
                dfuts.push_back(c.node);
            }
        }
        for (auto f : dfuts) {
            const int32_t c0 = S.nodes[f].child0;
            next_d.push_back({c0, false});
            next_d.push_back({c0 + 1, false});
        }
        dchecklist.swap(next_d);
        next_d.clear();
    }
    T.ref_stats[4] += nsink * S.lists[TGO_PC_D][n].size();
    T.ref_stats[0] += nsink * dsource_count;
    T.counts[2] += nsink * S.lists[TGO_PC_D][n].size();
    T.counts[0] += nsink * dsource_count;
    if (ewald) {
        echecklist.swap(next_e);
        next_e.clear();
        esource_count = 0;
        while (!echecklist.empty()) {
            efuts.clear();
            for (auto c : echecklist) {
                const Node &C = S.nodes[c.node];
                if (C.pe == C.pb) continue;
                const bool far = efar(C);
                if (c.opened) {
                    S.lists[TGO_PP_E][n].push_back(c.node);
                    esource_count += C.pe - C.pb;
                } else if (far) {
                    S.lists[TGO_PC_E][n].push_back(c.node);
                } else if (C.leaf()) {
                    c.opened = true;
                    next_e.push_back(c);
                } else {
                    efuts.push_back(c.node);
                }
            }
            for (auto f : efuts) {
                const int32_t c0 = S.nodes[f].child0;
                next_e.push_back({c0, false});
                next_e.push_back({c0 + 1, false});
            }
            echecklist.swap(next_e);
            next_e.clear();
        }
        T.ref_stats[5] += nsink * S.lists[TGO_PC_E][n].size();
        T.ref_stats[1] += nsink * esource_count;
        T.counts[3] += nsink * S.lists[TGO_PC_E][n].size();
        T.counts[1] += nsink * esource_count;
    }
}

void gather_multi(const Solver &S, const std::vector<int32_t> &ids, std::vector<float> &ym, std::vector<int32_t> &yx) {
    ym.resize(ids.size() * MP);
    yx.resize(ids.size() * 3);
    for (size_t k = 0; k < ids.size(); k++) {
        const Node &c = S.nodes[ids[k]];
        std::memcpy(&ym[k * MP], c.m, sizeof(float) * MP);
        for (int d = 0; d < 3; d++) yx[3 * k + d] = c.x[d];
    }
}

void gather_parts(const Solver &S, const std::vector<int32_t> &ids, std::vector<int32_t> &y) {
    y.clear();
    for (auto id : ids) {
        const Node &c = S.nodes[id];
        y.insert(y.end(), S.x.begin() + 3 * c.pb, S.x.begin() + 3 * c.pe);
    }
}

template <class F>
void parallel_for(int64_t n, int nthreads, F &&fn) {
    if (nthreads <= 1 || n < 2) {
        for (int64_t i = 0; i < n; i++) fn(i);
        return;
    }
    std::atomic<int64_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) {
        th.emplace_back([&]() {
            for (;;) {
                const int64_t i = next.fetch_add(1);
                if (i >= n) break;
                fn(i);
            }
        });
    }
    for (auto &t : th) t.join();
}

} // namespace

extern "C" {

/* kick_fmm list generation on nthreads threads, as the reference runs it
 * (src/tree.cpp:510-515 forks both children as HPX tasks): the top of the
 * tree is walked level by level until there are enough subtrees, then the
 * subtrees are walked concurrently.  Every node's lists are still written by
 * one task in the serial order, so the lists equal tgo_walk's. */
int tgo_walk_mt(void *h, int nthreads) {
    Solver &S = *(Solver *)h;
    if (nthreads <= 1) return tgo_walk(h);
    for (int k = 0; k < TGO_NLIST; k++) S.lists[k].assign(S.nodes.size(), std::vector<int32_t>());
    Tally total;
    std::vector<WalkTask> frontier;
    frontier.push_back({0, {{0, false}}, {{0, false}}});
    while (!frontier.empty() && frontier.size() < (size_t)(64 * nthreads)) {
        std::vector<WalkTask> next;
        for (auto &t : frontier) walk_node(S, t.node, std::move(t.d), std::move(t.e), total, &next);
        frontier.swap(next);
    }
    std::mutex mtx;
    parallel_for((int64_t)frontier.size(), nthreads, [&](int64_t k) {
        Tally T;
        WalkTask &t = frontier[k];
        walk_node(S, t.node, std::move(t.d), std::move(t.e), T, nullptr);
        std::lock_guard<std::mutex> lk(mtx);
        total.add(T);
    });
    for (int k = 0; k < 6; k++) S.ref_stats[k] = total.ref_stats[k];
    for (int k = 0; k < 8; k++) S.counts[k] = total.counts[k];
    return 0;
}

int tgo_load_reference(void *h, const char *so_path) {
    Solver &S = *(Solver *)h;
    if (S.dl) return 0;
    S.dl = dlopen(so_path, RTLD_NOW | RTLD_LOCAL);
    if (!S.dl) {
        fprintf(stderr, "tgo_load_reference: %s\n", dlerror());
        return -1;
    }
    auto init = (ref_init_fn)dlsym(S.dl, "ref_init");
    S.ref_pp_d = (tgo_pp_fn)dlsym(S.dl, "ref_PP_direct");
    S.ref_pc_d = (tgo_pc_fn)dlsym(S.dl, "ref_PC_direct");
    S.ref_cc_d = (tgo_cc_fn)dlsym(S.dl, "ref_CC_direct");
    S.ref_cp_d = (tgo_cp_fn)dlsym(S.dl, "ref_CP_direct");
    S.ref_pp_e = (tgo_pp_fn)dlsym(S.dl, "ref_PP_ewald");
    S.ref_pc_e = (tgo_pc_fn)dlsym(S.dl, "ref_PC_ewald");
    S.ref_cc_e = (tgo_cc_fn)dlsym(S.dl, "ref_CC_ewald");
    S.ref_cp_e = (tgo_cp_fn)dlsym(S.dl, "ref_CP_ewald");
    if (!init || !S.ref_pp_d || !S.ref_pc_d || !S.ref_cc_d || !S.ref_cp_d || !S.ref_pp_e || !S.ref_pc_e ||
        !S.ref_cc_e || !S.ref_cp_e)
        return -2;
    init(S.p.theta, S.p.soft_len, S.p.m * (double)S.n, (uint64_t)S.n, S.p.ewald, S.p.G);
    return 0;
}

/* Evaluation along the lists in the reference's order: per node
 * L = L_parent << (x - x_parent), then CC_direct, CP_direct, CC_ewald,
 * CP_ewald (src/tree.cpp:400-494); per leaf L2P then PC_direct, PP_direct,
 * PC_ewald, PP_ewald (src/tree.cpp:603-629). */
int tgo_evaluate(void *h, int use_ref, int nthreads, const int32_t *leaf_subset, int64_t nsubset) {
    Solver &S = *(Solver *)h;
    if (use_ref == 1 && !S.dl) return -1;
    tgo_pp_fn pp_d = tgo_PP_direct, pp_e = tgo_PP_ewald;
    tgo_pc_fn pc_d = tgo_PC_direct, pc_e = tgo_PC_ewald;
    tgo_cc_fn cc_d = tgo_CC_direct, cc_e = tgo_CC_ewald;
    tgo_cp_fn cp_d = tgo_CP_direct, cp_e = tgo_CP_ewald;
    if (use_ref == 1) {
        pp_d = S.ref_pp_d; pp_e = S.ref_pp_e; pc_d = S.ref_pc_d; pc_e = S.ref_pc_e;
        cc_d = S.ref_cc_d; cc_e = S.ref_cc_e; cp_d = S.ref_cp_d; cp_e = S.ref_cp_e;
    } else if (use_ref == 2) {
        pp_d = tgo64_PP_direct; pp_e = tgo64_PP_ewald; pc_d = tgo64_PC_direct; pc_e = tgo64_PC_ewald;
        cc_d = tgo64_CC_direct; cc_e = tgo64_CC_ewald; cp_d = tgo64_CP_direct; cp_e = tgo64_CP_ewald;
    }
    const size_t nn = S.nodes.size();
    S.L.assign(nn * LP, 0.0);
    S.f.assign(S.n * 4, 0.0);
    S.flops = S.p2m_flops;
    std::vector<char> active(nn, leaf_subset ? 0 : 1);
    std::vector<int32_t> leaves;
    if (leaf_subset) {
        for (int64_t k = 0; k < nsubset; k++) {
            int32_t i = leaf_subset[k];
            if (i < 0 || (size_t)i >= nn || !S.nodes[i].leaf()) return -3;
            leaves.push_back(i);
            while (i >= 0 && !active[i]) {
                active[i] = 1;
                i = S.nodes[i].parent;
            }
        }
    } else {
        for (size_t i = 0; i < nn; i++)
            if (S.nodes[i].leaf()) leaves.push_back((int32_t)i);
    }
    const bool ewald = S.p.ewald != 0;
    /* per level, parents before children */
    size_t b = 0;
    while (b < nn) {
        size_t e = b;
        while (e < nn && S.nodes[e].level == S.nodes[b].level) e++;
        parallel_for((int64_t)(e - b), nthreads, [&](int64_t k) {
            const size_t i = b + k;
            const Node &nd = S.nodes[i];
            if (!active[i] || nd.pe == nd.pb) return;
            double *L = &S.L[i * LP];
            double Lcom[3] = {0.5, 0.5, 0.5};
            if (nd.parent >= 0) {
                std::memcpy(L, &S.L[nd.parent * LP], sizeof(double) * LP);
                for (int d = 0; d < 3; d++) Lcom[d] = pos_to_double(S.nodes[nd.parent].x[d]);
            }
            double dx[3];
            for (int d = 0; d < 3; d++) dx[d] = pos_to_double(nd.x[d]) - Lcom[d];
            tgo_L2L(L, dx);
            std::vector<float> ym;
            std::vector<int32_t> yx, y;
            uint64_t fl = 0;
            gather_multi(S, S.lists[TGO_CC_D][i], ym, yx);
            fl += cc_d(&S.p, L, nd.x, ym.data(), yx.data(), (int)S.lists[TGO_CC_D][i].size());
            gather_parts(S, S.lists[TGO_CP_D][i], y);
            fl += cp_d(&S.p, L, nd.x, y.data(), (int)(y.size() / 3));
            if (ewald) {
                gather_multi(S, S.lists[TGO_CC_E][i], ym, yx);
                fl += cc_e(&S.p, L, nd.x, ym.data(), yx.data(), (int)S.lists[TGO_CC_E][i].size());
                gather_parts(S, S.lists[TGO_CP_E][i], y);
                fl += cp_e(&S.p, L, nd.x, y.data(), (int)(y.size() / 3));
            }
            S.flops += fl;
        });
        b = e;
    }
    parallel_for((int64_t)leaves.size(), nthreads, [&](int64_t k) {
        const int32_t i = leaves[k];
        const Node &nd = S.nodes[i];
        if (nd.pe == nd.pb) return;
        const int nx = (int)(nd.pe - nd.pb);
        const int32_t *xs = &S.x[3 * nd.pb];
        double *f = &S.f[4 * nd.pb];
        const double X[3] = {pos_to_double(nd.x[0]), pos_to_double(nd.x[1]), pos_to_double(nd.x[2])};
        for (int j = 0; j < nx; j++) {
            double dx[3];
            for (int d = 0; d < 3; d++) dx[d] = (double)(float)(pos_to_double(xs[3 * j + d]) - X[d]);
            tgo_L2P(&S.L[i * LP], dx, f + 4 * j);
        }
        std::vector<float> ym;
        std::vector<int32_t> yx, y;
        uint64_t fl = 0;
        gather_multi(S, S.lists[TGO_PC_D][i], ym, yx);
        fl += pc_d(&S.p, f, xs, nx, ym.data(), yx.data(), (int)S.lists[TGO_PC_D][i].size());
        gather_parts(S, S.lists[TGO_PP_D][i], y);
        fl += pp_d(&S.p, f, xs, nx, y.data(), (int)(y.size() / 3), 1);
        if (ewald) {
            gather_multi(S, S.lists[TGO_PC_E][i], ym, yx);
            fl += pc_e(&S.p, f, xs, nx, ym.data(), yx.data(), (int)S.lists[TGO_PC_E][i].size());
            gather_parts(S, S.lists[TGO_PP_E][i], y);
            fl += pp_e(&S.p, f, xs, nx, y.data(), (int)(y.size() / 3), 1);
        }
        S.flops += fl;
    });
    return 0;
}

/* Throughput of each interaction kind on the host, for the CPU baseline of a
 * workload too large to evaluate in full: for kind k (TGO_CC_D ... TGO_PP_E)
 * the kernel of that kind alone runs over randomly chosen sinks with a
 * non-empty list of that kind, on nthreads threads, until budget_s seconds or
 * all such sinks are done.  ns_per[k] = wall ns / interactions evaluated
 * (interactions counted as in tgo_get_stats), done[k] = interactions
 * evaluated.  A whole evaluation then costs about sum_k count_k * ns_per[k]. */
int tgo_kind_costs(void *h, int use_ref, int nthreads, double budget_s, uint64_t seed, double *ns_per, uint64_t *done) {
    Solver &S = *(Solver *)h;
    if (use_ref == 1 && !S.dl) return -1;
    const size_t nn = S.nodes.size();
    if (S.lists[0].size() != nn) return -2; /* no walk yet */
    const int nt = nthreads > 0 ? nthreads : 1;
    for (int kind = 0; kind < TGO_NLIST; kind++) {
        ns_per[kind] = 0.0;
        done[kind] = 0;
        std::vector<int32_t> sinks;
        for (size_t i = 0; i < nn; i++)
            if (!S.lists[kind][i].empty() && S.nodes[i].pe > S.nodes[i].pb) sinks.push_back((int32_t)i);
        if (sinks.empty()) continue;
        uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull + (uint64_t)kind;
        for (size_t a = sinks.size() - 1; a > 0; a--) { /* Fisher-Yates */
            st = st * 6364136223846793005ull + 1442695040888963407ull;
            std::swap(sinks[a], sinks[(size_t)((st >> 33) % (a + 1))]);
        }
        const bool node_kind = kind == TGO_CC_D || kind == TGO_CP_D || kind == TGO_CC_E || kind == TGO_CP_E;
        std::atomic<int64_t> next{0};
        std::atomic<uint64_t> work{0};
        std::atomic<bool> stop{false};
        const auto t0 = std::chrono::steady_clock::now();
        auto body = [&]() {
            std::vector<float> ym;
            std::vector<int32_t> yx, y;
            std::vector<double> f, L(LP);
            for (;;) {
                if (stop.load(std::memory_order_relaxed)) break;
                const int64_t k = next.fetch_add(1);
                if (k >= (int64_t)sinks.size()) break;
                const Node &nd = S.nodes[sinks[k]];
                const auto &lst = S.lists[kind][sinks[k]];
                const int nx = (int)(nd.pe - nd.pb);
                const int32_t *xs = &S.x[3 * nd.pb];
                uint64_t w = 0;
                if (node_kind) {
                    std::fill(L.begin(), L.end(), 0.0);
                    if (kind == TGO_CC_D || kind == TGO_CC_E) {
                        gather_multi(S, lst, ym, yx);
                        if (use_ref == 1)
                            (kind == TGO_CC_D ? S.ref_cc_d : S.ref_cc_e)(&S.p, L.data(), nd.x, ym.data(), yx.data(), (int)lst.size());
                        else
                            (kind == TGO_CC_D ? tgo_CC_direct : tgo_CC_ewald)(&S.p, L.data(), nd.x, ym.data(), yx.data(), (int)lst.size());
                        w = lst.size();
                    } else {
                        gather_parts(S, lst, y);
                        if (use_ref == 1)
                            (kind == TGO_CP_D ? S.ref_cp_d : S.ref_cp_e)(&S.p, L.data(), nd.x, y.data(), (int)(y.size() / 3));
                        else
                            (kind == TGO_CP_D ? tgo_CP_direct : tgo_CP_ewald)(&S.p, L.data(), nd.x, y.data(), (int)(y.size() / 3));
                        w = y.size() / 3;
                    }
                } else {
                    f.assign(4 * (size_t)nx, 0.0);
                    if (kind == TGO_PC_D || kind == TGO_PC_E) {
                        gather_multi(S, lst, ym, yx);
                        if (use_ref == 1)
                            (kind == TGO_PC_D ? S.ref_pc_d : S.ref_pc_e)(&S.p, f.data(), xs, nx, ym.data(), yx.data(), (int)lst.size());
                        else
                            (kind == TGO_PC_D ? tgo_PC_direct : tgo_PC_ewald)(&S.p, f.data(), xs, nx, ym.data(), yx.data(), (int)lst.size());
                        w = (uint64_t)nx * lst.size();
                    } else {
                        gather_parts(S, lst, y);
                        if (use_ref == 1)
                            (kind == TGO_PP_D ? S.ref_pp_d : S.ref_pp_e)(&S.p, f.data(), xs, nx, y.data(), (int)(y.size() / 3), 1);
                        else
                            (kind == TGO_PP_D ? tgo_PP_direct : tgo_PP_ewald)(&S.p, f.data(), xs, nx, y.data(), (int)(y.size() / 3), 1);
                        w = (uint64_t)nx * (y.size() / 3);
                    }
                }
                work.fetch_add(w);
                const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                if (el > budget_s) stop.store(true);
            }
        };
        std::vector<std::thread> th;
        for (int t = 0; t < nt; t++) th.emplace_back(body);
        for (auto &t : th) t.join();
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        done[kind] = work.load();
        ns_per[kind] = done[kind] ? el * 1e9 / (double)done[kind] : 0.0;
    }
    return 0;
}

int64_t tgo_num_nodes(void *h) { return (int64_t)((Solver *)h)->nodes.size(); }
int64_t tgo_num_particles(void *h) { return ((Solver *)h)->n; }

int tgo_get_nodes(void *h, uint64_t *boxid, int32_t *level, int64_t *pbegin, int64_t *pend, int32_t *child0,
                  int32_t *parent, int32_t *x, float *r, float *rmax, float *m) {
    Solver &S = *(Solver *)h;
    for (size_t i = 0; i < S.nodes.size(); i++) {
        const Node &nd = S.nodes[i];
        if (boxid) boxid[i] = nd.boxid;
        if (level) level[i] = nd.level;
        if (pbegin) pbegin[i] = nd.pb;
        if (pend) pend[i] = nd.pe;
        if (child0) child0[i] = nd.child0;
        if (parent) parent[i] = nd.parent;
        if (x)
            for (int d = 0; d < 3; d++) x[3 * i + d] = nd.x[d];
        if (r) r[i] = nd.r;
        if (rmax) rmax[i] = nd.rmax;
        if (m) std::memcpy(m + MP * i, nd.m, sizeof(float) * MP);
    }
    return 0;
}

int tgo_get_perm(void *h, int64_t *perm) {
    Solver &S = *(Solver *)h;
    std::memcpy(perm, S.perm.data(), sizeof(int64_t) * S.n);
    return 0;
}

int64_t tgo_list_size(void *h, int kind) {
    Solver &S = *(Solver *)h;
    if (kind < 0 || kind >= TGO_NLIST) return -1;
    int64_t tot = 0;
    for (auto &l : S.lists[kind]) tot += l.size();
    return tot;
}

int tgo_get_list(void *h, int kind, int64_t *offsets, int32_t *ids) {
    Solver &S = *(Solver *)h;
    if (kind < 0 || kind >= TGO_NLIST) return -1;
    int64_t o = 0;
    for (size_t i = 0; i < S.nodes.size(); i++) {
        offsets[i] = o;
        const auto &l = S.lists[kind][i];
        if (ids) std::memcpy(ids + o, l.data(), sizeof(int32_t) * l.size());
        o += l.size();
    }
    offsets[S.nodes.size()] = o;
    return 0;
}

int tgo_get_forces(void *h, double *phi, double *g) {
    Solver &S = *(Solver *)h;
    if ((int64_t)S.f.size() != 4 * S.n) return -1;
    for (int64_t i = 0; i < S.n; i++) {
        const int64_t c = S.perm[i];
        if (phi) phi[c] = S.f[4 * i];
        if (g)
            for (int d = 0; d < 3; d++) g[3 * c + d] = S.f[4 * i + 1 + d];
    }
    return 0;
}

int tgo_get_expansions(void *h, double *L) {
    Solver &S = *(Solver *)h;
    std::memcpy(L, S.L.data(), sizeof(double) * S.L.size());
    return 0;
}

int tgo_get_stats(void *h, uint64_t ref_stats[6], uint64_t counts[8], uint64_t *flops) {
    Solver &S = *(Solver *)h;
    if (ref_stats) std::memcpy(ref_stats, S.ref_stats, sizeof(S.ref_stats));
    if (counts) std::memcpy(counts, S.counts, sizeof(S.counts));
    if (flops) *flops = S.flops.load();
    return 0;
}

/* clean kick: v = v + float(g * (dt * G)) (src/part_vect.cpp:364,378) */
int tgo_kick(void *h, double dt) {
    Solver &S = *(Solver *)h;
    if ((int64_t)S.f.size() != 4 * S.n) return -1;
    for (int64_t i = 0; i < S.n; i++)
        for (int d = 0; d < 3; d++) S.v[3 * i + d] = S.v[3 * i + d] + (float)(S.f[4 * i + 1 + d] * (dt * S.p.G));
    return 0;
}

/* part_vect_drift (src/part_vect.cpp:493-540), non-cosmological */
int tgo_drift(void *h, double dt, double *ekin) {
    Solver &S = *(Solver *)h;
    double ek = 0.0;
    const float fdt = (float)dt;
    for (int64_t i = 0; i < S.n; i++) {
        const float *v = &S.v[3 * i];
        ek += 0.5 * S.p.m * (double)(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int d = 0; d < 3; d++) {
            double xx = pos_to_double(S.x[3 * i + d]);
            xx += (double)(v[d] * fdt);
            while (xx >= 1.0) xx -= 1.0;
            while (xx < 0.0) xx += 1.0;
            S.x[3 * i + d] = double_to_pos(xx);
        }
    }
    if (ekin) *ekin = ek;
    return 0;
}

int tgo_get_particles(void *h, int32_t *x, float *v) {
    Solver &S = *(Solver *)h;
    for (int64_t i = 0; i < S.n; i++) {
        const int64_t c = S.perm[i];
        for (int d = 0; d < 3; d++) {
            if (x) x[3 * c + d] = S.x[3 * i + d];
            if (v) v[3 * c + d] = S.v[3 * i + d];
        }
    }
    return 0;
}

int tgo_energy(void *h, double out[5]) {
    Solver &S = *(Solver *)h;
    double ek = 0, ep = 0, p[3] = {0, 0, 0};
    for (int64_t i = 0; i < S.n; i++) {
        const float *v = &S.v[3 * i];
        double v2 = 0;
        for (int d = 0; d < 3; d++) {
            v2 += (double)v[d] * v[d];
            p[d] += (double)v[d] / (double)S.n;
        }
        ek += 0.5 * S.p.m * v2;
        if ((int64_t)S.f.size() == 4 * S.n) ep += 0.5 * S.p.m * S.f[4 * i] * S.p.G;
    }
    out[0] = ek;
    out[1] = ep;
    out[2] = p[0];
    out[3] = p[1];
    out[4] = p[2];
    return 0;
}

/* ---------------- FP64 ground truth ---------------- */

/* Reference-convention correction (alpha = 2, green.hpp lattice sets) in double. */
void tgo_ewald_corr_f64(const double dx[3], double out[4]) {
    const double r = std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    if (r < 1e-6) {
        out[0] = 2.8372975;
        out[1] = out[2] = out[3] = 0.0;
        return;
    }
    double phi = 0, g[3] = {0, 0, 0};
    for (auto &nv : REAL_IDX.v) {
        const double d[3] = {dx[0] - nv[0], dx[1] - nv[1], dx[2] - nv[2]};
        const double rr = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (rr >= 3.6) continue;
        const double erfc = std::erfc(2.0 * rr);
        const double ef = 4.0 / std::sqrt(M_PI) * rr * std::exp(-4.0 * rr * rr);
        phi -= erfc / rr;
        const double d1 = (ef + erfc) / (rr * rr * rr);
        for (int a = 0; a < 3; a++) g[a] -= d[a] * d1;
    }
    for (auto &hv : FOUR_IDX.v) {
        const double h2 = (double)hv[0] * hv[0] + (double)hv[1] * hv[1] + (double)hv[2] * hv[2];
        if (h2 == 0) continue;
        const double c0 = std::exp(-M_PI * M_PI * h2 / 4.0) / h2;
        const double om = 2.0 * M_PI * (dx[0] * hv[0] + dx[1] * hv[1] + dx[2] * hv[2]);
        phi += -(1.0 / M_PI) * c0 * std::cos(om);
        for (int a = 0; a < 3; a++) g[a] -= 2.0 * hv[a] * c0 * std::sin(om);
    }
    phi += M_PI / 4.0 + 1.0 / r;
    for (int a = 0; a < 3; a++) g[a] += dx[a] / (r * r * r);
    out[0] = phi;
    for (int a = 0; a < 3; a++) out[1 + a] = g[a];
}

/* FP64 direct Ewald sum with split parameter alpha:
 *   psi(x) = -sum_n erfc(alpha|x-n|)/|x-n| - sum_{h!=0} exp(-pi^2 h^2/alpha^2)/(pi h^2) cos(2 pi h.x) + pi/alpha^2
 * (the reference's convention, tigergrav/green.hpp:30-59,189-286, for any alpha);
 * real-space images with alpha*|x-n| < 6.2, Fourier vectors with
 * pi^2 h^2/alpha^2 < 38 (truncation ~1e-16).  Fourier part by structure
 * factors.  Nearest-image pairs closer than h use the GADGET spline
 * (src/gravity.cpp:231-287) instead of 1/r; the self pair contributes the
 * r->0 limits (potential only). */
int tgo_truth(const int32_t *x, int64_t n, const int64_t *samples, int64_t ns, double m, double h, double alpha,
              int nthreads, double *phi_out, double *g_out) {
    if (n < 1 || alpha < 4.2) return -1; /* images beyond +-1 must fall outside 6.2/alpha */
    const double rcut_real = 6.2 / alpha;
    const double h2max = 38.0 * alpha * alpha / (M_PI * M_PI);
    const int hmax = (int)std::sqrt(h2max) + 1;
    std::vector<std::array<int, 3>> hv;
    for (int i = 0; i <= hmax; i++)
        for (int j = -hmax; j <= hmax; j++)
            for (int k = -hmax; k <= hmax; k++) {
                if (i == 0 && (j < 0 || (j == 0 && k <= 0))) continue; /* half space */
                if ((double)(i * i + j * j + k * k) < h2max) hv.push_back({i, j, k});
            }
    const size_t nh = hv.size();
    std::vector<double> Sc(nh, 0.0), Ss(nh, 0.0);
    /* structure factors, parallel over h */
    parallel_for((int64_t)nh, nthreads, [&](int64_t q) {
        double c = 0, s = 0;
        for (int64_t j = 0; j < n; j++) {
            const double om = 2.0 * M_PI *
                              (hv[q][0] * pos_to_double(x[3 * j]) + hv[q][1] * pos_to_double(x[3 * j + 1]) +
                               hv[q][2] * pos_to_double(x[3 * j + 2]));
            c += std::cos(om);
            s += std::sin(om);
        }
        Sc[q] = c;
        Ss[q] = s;
    });
    const double sqrtpi = std::sqrt(M_PI);
    parallel_for(ns, nthreads, [&](int64_t k) {
        const int64_t i = samples[k];
        double phi = 0, g[3] = {0, 0, 0};
        const double xi[3] = {pos_to_double(x[3 * i]), pos_to_double(x[3 * i + 1]), pos_to_double(x[3 * i + 2])};
        for (int64_t j = 0; j < n; j++) {
            double d[3];
            for (int a = 0; a < 3; a++) d[a] = (double)(int32_t)((uint32_t)x[3 * i + a] - (uint32_t)x[3 * j + a]) * POS_INV;
            for (int nx = -1; nx <= 1; nx++)
                for (int ny = -1; ny <= 1; ny++)
                    for (int nz = -1; nz <= 1; nz++) {
                        const double e[3] = {d[0] - nx, d[1] - ny, d[2] - nz};
                        const double r2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
                        const double r = std::sqrt(r2);
                        if (r >= rcut_real) continue;
                        const bool nearest = (nx == 0 && ny == 0 && nz == 0);
                        if (r == 0.0) {
                            /* self pair, n = 0: the regular part erf(alpha r)/r -> 2 alpha/sqrt(pi);
                             * then the softened self potential -14/5 m/h (src/gravity.cpp:280-286)
                             * and the phi_self term +315/128 m/h (src/gravity.cpp:187,295)  */
                            phi += m * (2.0 * alpha / sqrtpi);
                            phi += m * (-(14.0 / 5.0) / h + (315.0 / 128.0) / h);
                            continue;
                        }
                        const double erfc = std::erfc(alpha * r);
                        const double ef = 2.0 * alpha / sqrtpi * r * std::exp(-alpha * alpha * r2);
                        phi -= m * erfc / r;
                        double d1 = (ef + erfc) / (r2 * r);
                        if (nearest && r < h) {
                            /* replace the nearest-image 1/r by the softened kernel */
                            const double u = r / h;
                            double fk, pk;
                            if (u < 0.5) {
                                fk = (32.0 * u * u * u - 192.0 / 5.0 * u * u + 32.0 / 3.0) / (h * h * h);
                                pk = (-32.0 / 5.0 * u * u * u * u * u + 48.0 / 5.0 * u * u * u * u - 16.0 / 3.0 * u * u + 14.0 / 5.0) / h;
                            } else {
                                fk = (-32.0 / 3.0 * u * u * u + 192.0 / 5.0 * u * u - 48.0 * u + 64.0 / 3.0) / (h * h * h) -
                                     1.0 / (15.0 * r2 * r);
                                pk = (32.0 / 15.0 * u * u * u * u * u - 48.0 / 5.0 * u * u * u * u + 16.0 * u * u * u -
                                      32.0 / 3.0 * u * u + 16.0 / 5.0) / h - 1.0 / (15.0 * r);
                            }
                            d1 += fk - 1.0 / (r2 * r);
                            phi += m * (1.0 / r - pk);
                        }
                        for (int a = 0; a < 3; a++) g[a] -= m * e[a] * d1;
                    }
        }
        for (size_t q = 0; q < nh; q++) {
            const double hh = (double)(hv[q][0] * hv[q][0] + hv[q][1] * hv[q][1] + hv[q][2] * hv[q][2]);
            const double c0 = std::exp(-M_PI * M_PI * hh / (alpha * alpha)) / hh;
            const double om = 2.0 * M_PI * (hv[q][0] * xi[0] + hv[q][1] * xi[1] + hv[q][2] * xi[2]);
            const double ci = std::cos(om), si = std::sin(om);
            /* sum_j cos(om_i - om_j) = ci*C + si*S ; sum_j sin(om_i - om_j) = si*C - ci*S ; two half spaces */
            const double sc = ci * Sc[q] + si * Ss[q];
            const double ss = si * Sc[q] - ci * Ss[q];
            phi += 2.0 * m * (-(1.0 / M_PI) * c0 * sc);
            for (int a = 0; a < 3; a++) g[a] -= 2.0 * m * 2.0 * hv[q][a] * c0 * ss;
        }
        phi += m * (double)n * M_PI / (alpha * alpha);
        phi_out[k] = phi;
        for (int a = 0; a < 3; a++) g_out[3 * k + a] = g[a];
    });
    return 0;
}

} // extern "C"
