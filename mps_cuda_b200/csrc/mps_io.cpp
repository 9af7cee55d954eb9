// mps_io.cpp -- the reference's input files and its parameter derivation, on the host.
//
// MPS_physical.txt and initial.txt are what the reference's RdDat reads (kernel.cu:4-143);
// with these a scene prepared for the reference drops into this library unchanged. The
// parsing follows RdDat: every number of both files is read as a float (kernel.cu:12-22,
// 117-119) and then widened, walls (WLL) and moving walls (OBJ) store the negated file normal
// as their inward normal (kernel.cu:126-128), and particles outside the padded domain are
// dropped (kernel.cu:121). OBJ2 particles, whose normal the reference leaves unset, get the
// negated file normal too; fluid particles a zero normal.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <string>

#include "../../include/mps_b200.h"

namespace mps {
extern thread_local std::string g_last_error;
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
}  // namespace mps

namespace {

constexpr int kFLD = 0, kWLL = 1, kOBJ = 2, kOBJ2 = 3;

struct File {
    FILE* f;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

bool read_floats(FILE* f, float* v, int n) {
    for (int k = 0; k < n; ++k)
        if (std::fscanf(f, "%f", v + k) != 1) return false;
    return true;
}

}  // namespace

extern "C" {

int mps_read_physical(const char* path, mps_physical* out) {
    if (!path || !out) return mps::fail(MPS_ERR_ARG, "path and out must not be NULL");
    File in(path, "r");
    if (!in.f) return mps::fail(MPS_ERR_ARG, std::string("cannot open ") + path + ": " + std::strerror(errno));
    float s[17];
    if (!read_floats(in.f, s, 17))
        return mps::fail(MPS_ERR_ARG, std::string(path) + ": expected 17 numbers (kernel.cu:12-22)");
    std::memset(out, 0, sizeof(*out));
    for (int d = 0; d < 3; ++d) {
        out->min[d] = s[d];
        out->max[d] = s[3 + d];
        out->g[d] = s[6 + d];
    }
    out->fin_tim = s[9];
    out->output_time = s[10];
    out->mach = s[11];
    out->courant = s[12];
    out->col_rat = s[13];
    out->dst_lmt_rat = s[14];
    out->knm_vsc = s[15];
    out->pcl_dst = s[16];
    return MPS_OK;
}

int mps_write_physical(const char* path, const mps_physical* ph) {
    if (!path || !ph) return mps::fail(MPS_ERR_ARG, "path and ph must not be NULL");
    File f(path, "w");
    if (!f.f) return mps::fail(MPS_ERR_ARG, std::string("cannot create ") + path);
    // one line per group, as the reference's reads are grouped (kernel.cu:12-22)
    for (const double* v : {ph->min, ph->max, ph->g})
        std::fprintf(f.f, "%.17g %.17g %.17g\n", v[0], v[1], v[2]);
    std::fprintf(f.f, "%.17g\n%.17g\n%.17g\n%.17g\n%.17g\n%.17g\n%.17g\n%.17g\n", ph->fin_tim,
                 ph->output_time, ph->mach, ph->courant, ph->col_rat, ph->dst_lmt_rat,
                 ph->knm_vsc, ph->pcl_dst);
    return std::ferror(f.f) ? mps::fail(MPS_ERR_ARG, std::string("write failed: ") + path) : MPS_OK;
}

int mps_read_initial(const char* path, const mps_physical* ph, int32_t cap, int8_t* typ,
                     double* pos, double* nrm, int32_t* n_out) {
    if (!path || !ph || !n_out) return mps::fail(MPS_ERR_ARG, "path, ph and n_out must not be NULL");
    File in(path, "r");
    if (!in.f) return mps::fail(MPS_ERR_ARG, std::string("cannot open ") + path + ": " + std::strerror(errno));
    int np = 0;
    if (std::fscanf(in.f, "%d", &np) != 1 || np < 0)
        return mps::fail(MPS_ERR_ARG, std::string(path) + ": expected the particle count first");
    // padded domain, as RdDat computes it (kernel.cu:25-31) in the reference's float
    const float l0 = float(ph->pcl_dst);
    float lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = float(float(ph->min[d]) - 3.1 * l0);
        hi[d] = float(float(ph->max[d]) + 3.1 * l0);
    }
    int kept = 0;
    for (int i = 0; i < np; ++i) {
        int idx = 0, t = 0;
        float v[7];
        if (std::fscanf(in.f, " %d %d", &idx, &t) != 2 || !read_floats(in.f, v, 7))
            return mps::fail(MPS_ERR_ARG, std::string(path) + ": line " + std::to_string(i + 2) +
                                              " is not 'idx typ x y z nx ny nz g' (kernel.cu:117)");
        if (!(v[0] < hi[0] && v[0] > lo[0] && v[1] < hi[1] && v[1] > lo[1] && v[2] < hi[2] &&
              v[2] > lo[2]))
            continue;
        if (typ && pos && nrm && kept < cap) {
            typ[kept] = int8_t(t);
            bool wall = t == kWLL || t == kOBJ || t == kOBJ2;
            for (int d = 0; d < 3; ++d) {
                pos[size_t(d) * cap + kept] = double(v[d]);
                nrm[size_t(d) * cap + kept] = wall ? -double(v[3 + d]) : 0.0;
            }
        }
        ++kept;
    }
    *n_out = kept;
    if (kept > cap || !typ || !pos || !nrm)
        return mps::fail(MPS_ERR_ARG, std::to_string(kept) + " particles lie inside the padded domain; "
                                          "call again with cap >= *n");
    // the arrays are SoA with stride cap; pack them to stride n
    if (kept < cap)
        for (int d = 1; d < 3; ++d) {
            std::memmove(pos + size_t(d) * kept, pos + size_t(d) * cap, sizeof(double) * kept);
            std::memmove(nrm + size_t(d) * kept, nrm + size_t(d) * cap, sizeof(double) * kept);
        }
    return MPS_OK;
}

int mps_write_initial(const char* path, int32_t n, const int8_t* typ, const double* pos,
                      const double* nrm) {
    if (!path || n < 0 || (n > 0 && (!typ || !pos || !nrm)))
        return mps::fail(MPS_ERR_ARG, "path, typ, pos and nrm must be given");
    File f(path, "w");
    if (!f.f) return mps::fail(MPS_ERR_ARG, std::string("cannot create ") + path);
    std::fprintf(f.f, "%d\n", n);
    for (int i = 0; i < n; ++i) {
        // the file holds the outward normal: RdDat negates it (kernel.cu:126-128)
        const double s = (typ[i] == kFLD) ? 0.0 : -1.0;
        std::fprintf(f.f, "%d %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", i, int(typ[i]),
                     pos[i], pos[size_t(n) + i], pos[2 * size_t(n) + i], s * nrm[i] + 0.0,
                     s * nrm[size_t(n) + i] + 0.0, s * nrm[2 * size_t(n) + i] + 0.0, 0.0);
    }
    return std::ferror(f.f) ? mps::fail(MPS_ERR_ARG, std::string("write failed: ") + path) : MPS_OK;
}

int mps_params_from_physical(const mps_physical* ph, int32_t n, const int8_t* typ,
                             const double* pos, int32_t precision, mps_params* out) {
    if (!ph || !out || n < 0 || (n > 0 && (!typ || !pos)))
        return mps::fail(MPS_ERR_ARG, "ph, out, typ and pos must be given");
    if (!(ph->pcl_dst > 0) || !(ph->mach > 0))
        return mps::fail(MPS_ERR_ARG, "pcl_dst and the Mach number must be positive");
    // SetPara (kernel.cu:396-412) takes the fluid's extent and gravity along y; here the
    // axis is the one gravity points along, which is y for the reference's own scenes
    int ax = 0;
    for (int d = 1; d < 3; ++d)
        if (std::fabs(ph->g[d]) > std::fabs(ph->g[ax])) ax = d;
    double hmin = 1e300, hmax = -1e300;
    for (int i = 0; i < n; ++i)
        if (typ[i] == kFLD) {
            const double h = pos[size_t(ax) * n + i];
            hmin = std::fmin(hmin, h);
            hmax = std::fmax(hmax, h);
        }
    const double H = hmax > hmin ? hmax - hmin : 0.0;
    const double g = std::fabs(ph->g[ax]);
    std::memset(out, 0, sizeof(*out));
    out->pcl_dst = ph->pcl_dst;
    for (int d = 0; d < 3; ++d) {
        out->min[d] = ph->min[d];
        out->max[d] = ph->max[d];
        out->g[d] = ph->g[d];
    }
    out->knm_vsc = ph->knm_vsc;
    out->col_rat = ph->col_rat;
    out->dst_lmt_rat = ph->dst_lmt_rat;
    out->rho = 1000.0;                     // Dns_FLD (const.cuh:37)
    out->umax = std::sqrt(2.0 * g * H);    // kernel.cu:407
    out->snd = out->umax / ph->mach;       // kernel.cu:408
    out->pmax = out->rho * g * H;          // kernel.cu:411, with |g|
    out->dt = out->umax + out->snd > 0 ? ph->pcl_dst / (out->umax + out->snd) : 0.0;  // :415
    out->precision = precision;
    return MPS_OK;
}

}  // extern "C"
