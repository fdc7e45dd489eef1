/*
 * tg_load.cu -- N-GenIC / Gadget-1 initial conditions (load_header,
 * load_particles, src/load.cpp:13-96), host code behind the C ABI.
 *
 * File layout (Fortran records: int32 length before and after each block):
 * the 256-byte io_header_1 (tigergrav/load.hpp:20-39), then npart[1]
 * positions (3 floats each), then npart[1] velocities.  As the reference
 * does: positions are taken to be in box units, shifted by half the mean
 * spacing 0.5 N^(-1/3) in FP32, wrapped with `while (x > 1) x -= 1`, and
 * converted with double_to_pos; velocities are scaled by a^1.5 with
 * a = 1 / (1 + redshift).  Other particle types are ignored.
 */
#include <cmath>
#include <cstdio>
#include <cstring>

namespace tg {

#pragma pack(push, 4)
struct GadgetHeader1 {
    uint32_t npart[6];
    double mass[6];
    double time;
    double redshift;
    int32_t flag_sfr;
    int32_t flag_feedback;
    uint32_t npartTotal[6];
    int32_t flag_cooling;
    int32_t num_files;
    double BoxSize;
    double Omega0;
    double OmegaLambda;
    double HubbleParam;
    int32_t flag_stellarage;
    int32_t flag_metals;
    int32_t hashtabsize;
    char fill[84];
};
#pragma pack(pop)
static_assert(sizeof(GadgetHeader1) == 256, "io_header_1 is 256 bytes");

/* double_to_pos (tigergrav/position.hpp:30-37): lround((x - 0.5) 2^32), wrapped */
static int32_t host_double_to_pos(double x) {
    long long z = std::llround((x - 0.5) * 4294967296.0);
    if ((double)z >= 2147483648.0) z -= 4294967296ll;
    return (int32_t)z;
}

static bool read_record(FILE *fp, void *dst, size_t bytes) {
    int32_t len0 = 0, len1 = 0;
    if (fread(&len0, 4, 1, fp) != 1) return false;
    if (dst && fread(dst, 1, bytes, fp) != bytes) return false;
    if (!dst && fseek(fp, (long)bytes, SEEK_CUR) != 0) return false;
    if (fread(&len1, 4, 1, fp) != 1) return false;
    return true;
}

} // namespace tg

/* header -> (npart[1], redshift, mass[1], Omega0, OmegaLambda, HubbleParam, BoxSize, time) */
extern "C" int tg_load_gadget1(const char *path, double *header, int32_t *x, float *v, int64_t capacity,
                               int64_t *n_out) {
    if (!path || !n_out) return TG_ERR_ARG;
    FILE *fp = fopen(path, "rb");
    if (!fp) return TG_ERR_ARG;
    tg::GadgetHeader1 h;
    if (!tg::read_record(fp, &h, sizeof(h))) {
        fclose(fp);
        return TG_ERR_ARG;
    }
    const int64_t n = h.npart[1];
    *n_out = n;
    if (header) {
        const double vals[8] = {(double)n, h.redshift, h.mass[1], h.Omega0, h.OmegaLambda, h.HubbleParam,
                                h.BoxSize, h.time};
        std::memcpy(header, vals, sizeof(vals));
    }
    if (!x) {
        fclose(fp);
        return TG_OK;
    }
    if (capacity < n) {
        fclose(fp);
        return TG_ERR_SIZE;
    }
    int32_t len = 0;
    int rc = TG_OK;
    if (fread(&len, 4, 1, fp) != 1) rc = TG_ERR_ARG;
    const double sep = 0.5 * std::pow((double)n, -1.0 / 3.0);
    for (int64_t i = 0; rc == TG_OK && i < n; i++) {
        float p[3];
        if (fread(p, sizeof(float), 3, fp) != 3) {
            rc = TG_ERR_ARG;
            break;
        }
        for (int d = 0; d < 3; d++) {
            float c = p[d];
            c += sep; /* float += double, as src/load.cpp:62-64 */
            while (c > 1.0) c -= 1.0;
            x[3 * i + d] = tg::host_double_to_pos(c);
        }
    }
    if (rc == TG_OK && fread(&len, 4, 1, fp) != 1) rc = TG_ERR_ARG;
    if (rc == TG_OK && v) {
        if (fread(&len, 4, 1, fp) != 1) rc = TG_ERR_ARG;
        const double c0 = 1.0 / (1.0 + h.redshift);
        const double s = std::pow(c0, 1.5);
        for (int64_t i = 0; rc == TG_OK && i < n; i++) {
            float q[3];
            if (fread(q, sizeof(float), 3, fp) != 3) {
                rc = TG_ERR_ARG;
                break;
            }
            for (int d = 0; d < 3; d++) v[3 * i + d] = (float)(q[d] * s);
        }
    }
    fclose(fp);
    return rc;
}
