/*
 * ref_driver.cpp -- C wrappers around the reference's own gravity kernels.
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `ref`) against
 * the reference sources where they lie (src/gravity.cpp and its headers),
 * never copied; output goes to oracle/_ref/.  The reference keeps its
 * parameters in a global options object (tigergrav/options.hpp:79-82) whose
 * definition lives in src/options.cpp (needs Boost/HPX); this file supplies
 * that definition.  The kernels cache options in function-local statics on
 * first use (e.g. src/gravity.cpp:176-187), so ref_init must run once, before
 * any kernel, and later calls must repeat the same parameters.
 */
#include <tigergrav/gravity.hpp>
#include <tigergrav/green.hpp>
#include <tigergrav/options.hpp>

#include <cstring>
#include <vector>

#include "tg_oracle.h"

options options::global;
options &options::get() { return global; }
void options::set(options o) { global = o; }

static bool g_inited = false;
static double g_key[6];

extern "C" int ref_init(double theta, double soft_len, double m_tot, uint64_t n, int ewald, double G) {
    const double key[6] = {theta, soft_len, m_tot, (double)n, (double)ewald, G};
    if (g_inited) return std::memcmp(key, g_key, sizeof(key)) == 0 ? 0 : -1;
    options o = options();
    o.theta = theta;
    o.soft_len = soft_len;
    o.m_tot = m_tot;
    o.problem_size = n;
    o.ewald = ewald != 0;
    o.G = G;
    o.parts_per_node = 64;
    o.cosmic = false;
    o.glass = false;
    options::set(o);
    std::memcpy(g_key, key, sizeof(key));
    g_inited = true;
    return 0;
}

static std::vector<force> to_forces(const double *f, int nx) {
    std::vector<force> F(nx);
    for (int i = 0; i < nx; i++) {
        F[i].phi = f[4 * i];
        for (int d = 0; d < 3; d++) F[i].g[d] = f[4 * i + 1 + d];
    }
    return F;
}
static void from_forces(const std::vector<force> &F, double *f) {
    for (size_t i = 0; i < F.size(); i++) {
        f[4 * i] = F[i].phi;
        for (int d = 0; d < 3; d++) f[4 * i + 1 + d] = F[i].g[d];
    }
}
static std::vector<vect<pos_type>> to_pos(const int32_t *x, int n) {
    std::vector<vect<pos_type>> X(n);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) X[i][d] = x[3 * i + d];
    return X;
}
static std::vector<multi_src> to_multi(const float *ym, const int32_t *yx, int n) {
    std::vector<multi_src> Y(n);
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < MP; k++) Y[i].m[k] = ym[MP * i + k];
        for (int d = 0; d < 3; d++) Y[i].x[d] = yx[3 * i + d];
    }
    return Y;
}
static expansion<double> to_exp(const double *L) {
    expansion<double> E;
    for (int i = 0; i < LP; i++) E[i] = L[i];
    return E;
}
static void from_exp(const expansion<double> &E, double *L) {
    for (int i = 0; i < LP; i++) L[i] = E[i];
}

#define PP_WRAP(NAME, CALL)                                                                            \
    extern "C" uint64_t ref_##NAME(const tgo_params *, double *f, const int32_t *x, int nx, const int32_t *y, \
                                   int ny, int do_phi) {                                              \
        auto F = to_forces(f, nx);                                                                     \
        auto X = to_pos(x, nx);                                                                        \
        auto Y = to_pos(y, ny);                                                                        \
        (void)do_phi;                                                                                  \
        const uint64_t fl = CALL;                                                                      \
        from_forces(F, f);                                                                             \
        return fl;                                                                                     \
    }
PP_WRAP(PP_direct, gravity_PP_direct(F, X, Y, do_phi != 0))
PP_WRAP(PP_ewald, gravity_PP_ewald(F, X, Y))

#define PC_WRAP(NAME, FN)                                                                              \
    extern "C" uint64_t ref_##NAME(const tgo_params *, double *f, const int32_t *x, int nx, const float *ym, \
                                   const int32_t *yx, int ny) {                                       \
        auto F = to_forces(f, nx);                                                                     \
        auto X = to_pos(x, nx);                                                                        \
        auto Y = to_multi(ym, yx, ny);                                                                 \
        const uint64_t fl = FN(F, X, Y);                                                               \
        from_forces(F, f);                                                                             \
        return fl;                                                                                     \
    }
PC_WRAP(PC_direct, gravity_PC_direct)
PC_WRAP(PC_ewald, gravity_PC_ewald)

#define CC_WRAP(NAME, FN)                                                                              \
    extern "C" uint64_t ref_##NAME(const tgo_params *, double *L, const int32_t *x, const float *ym,       \
                                   const int32_t *yx, int ny) {                                       \
        auto E = to_exp(L);                                                                            \
        vect<pos_type> X;                                                                              \
        for (int d = 0; d < 3; d++) X[d] = x[d];                                                       \
        auto Y = to_multi(ym, yx, ny);                                                                 \
        const uint64_t fl = FN(E, X, Y);                                                               \
        from_exp(E, L);                                                                                \
        return fl;                                                                                     \
    }
CC_WRAP(CC_direct, gravity_CC_direct)
CC_WRAP(CC_ewald, gravity_CC_ewald)

#define CP_WRAP(NAME, FN)                                                                              \
    extern "C" uint64_t ref_##NAME(const tgo_params *, double *L, const int32_t *x, const int32_t *y,     \
                                   int ny) {                                                          \
        auto E = to_exp(L);                                                                            \
        vect<pos_type> X;                                                                              \
        for (int d = 0; d < 3; d++) X[d] = x[d];                                                       \
        auto Y = to_pos(y, ny);                                                                        \
        const uint64_t fl = FN(E, X, Y);                                                               \
        from_exp(E, L);                                                                                \
        return fl;                                                                                     \
    }
CP_WRAP(CP_direct, gravity_CP_direct)
CP_WRAP(CP_ewald, gravity_CP_ewald)

/* the reference's own expansion algebra, for pinning the restatement */
extern "C" void ref_green_ewald(const float dx[3], float D[35]) {
    vect<simd_float> X;
    for (int d = 0; d < 3; d++) X[d] = simd_float(dx[d]);
    const auto E = green_ewald(X);
    for (int i = 0; i < LP; i++) D[i] = E[i][0];
}
extern "C" void ref_green_direct(const float dx[3], float D[35]) {
    vect<simd_float> X;
    for (int d = 0; d < 3; d++) X[d] = simd_float(dx[d]);
    const auto E = green_direct(X);
    for (int i = 0; i < LP; i++) D[i] = E[i][0];
}
extern "C" void ref_L2L(double L[35], const double dx[3]) {
    auto E = to_exp(L);
    vect<double> X;
    for (int d = 0; d < 3; d++) X[d] = dx[d];
    E <<= X;
    from_exp(E, L);
}
extern "C" void ref_L2P(const double L[35], const double dx[3], double out[4]) {
    auto E = to_exp(L);
    vect<double> X;
    for (int d = 0; d < 3; d++) X[d] = dx[d];
    const force f = E.translate_L2(X);
    out[0] = f.phi;
    for (int d = 0; d < 3; d++) out[1 + d] = f.g[d];
}
extern "C" void ref_M2M(float M[17], const float dx[3]) {
    multipole<float> m;
    for (int i = 0; i < MP; i++) m[i] = M[i];
    vect<float> X;
    for (int d = 0; d < 3; d++) X[d] = dx[d];
    m >>= X;
    for (int i = 0; i < MP; i++) M[i] = m[i];
}
