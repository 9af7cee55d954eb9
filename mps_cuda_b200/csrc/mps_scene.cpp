// mps_scene.cpp -- dam-break scene generator (host only).
//
// The reference reads its particles from initial.txt (kernel.cu:59-141): one line per
// particle with type, position and wall normal. No such file ships with it, so scenes are
// generated here: a rectangular tank whose faces each carry one layer of wall particles on
// the face plane at in-plane positions ((p+1/2) l0, (q+1/2) l0), and a fluid block on the
// lattice ((i+1/2) l0, (j+1/2) l0, (k+1/2) l0) with a uniform jitter. Where two faces meet,
// their first rows lie l0/sqrt(2) apart with different normals, so Surface_Edge
// (kernel.cu:580-581, dist2 < l0^2) marks exactly those rows as Edge; no two wall particles
// share a position and no wall distance sits near that threshold, so neither the edge test
// nor the nearest-wall choice of MRRinout (kernel.cu:965-971) depends on visiting order or
// rounding. Normals are the reference's WLLVec: unit vectors pointing into the tank.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>

#include "../../include/mps_b200.h"

namespace {

// 53-bit uniform in [0, 1) from one mt19937_64 draw
double u01(std::mt19937_64& g) { return double(g() >> 11) * (1.0 / 9007199254740992.0); }

// Box-Muller standard normals, generated in pairs
struct Normal {
    std::mt19937_64 g;
    bool have = false;
    double spare = 0;
    explicit Normal(uint64_t seed) : g(seed) {}
    double next() {
        if (have) { have = false; return spare; }
        double u1 = u01(g), u2 = u01(g);
        if (u1 <= 0) u1 = 1.0 / 9007199254740992.0;
        double rad = std::sqrt(-2.0 * std::log(u1)), th = 6.283185307179586 * u2;
        spare = rad * std::sin(th);
        have = true;
        return rad * std::cos(th);
    }
};

int face_points(const mps_scene_desc& d, int face, int n[3]) {
    // points per axis: L / l0 cells, one particle at the centre of each
    for (int a = 0; a < 3; ++a) n[a] = int(std::lround(d.tank[a] / d.l0));
    int axis = face / 2;
    int cnt = 1;
    for (int a = 0; a < 3; ++a)
        if (a != axis) cnt *= n[a];
    return cnt;
}

bool valid(const mps_scene_desc* d) {
    if (!d || !(d->l0 > 0)) return false;
    for (int a = 0; a < 3; ++a)
        if (!(d->tank[a] > 0) || d->block[a] < 0) return false;
    return true;
}

}  // namespace

extern "C" {

int mps_scene_dambreak_count(const mps_scene_desc* d, int32_t* n_out) {
    if (!valid(d) || !n_out) return MPS_ERR_ARG;
    long long n = (long long)d->block[0] * d->block[1] * d->block[2];
    for (int f = 0; f < 6; ++f) {
        if (!(d->wall_mask & (1 << f))) continue;
        int nn[3];
        n += face_points(*d, f, nn);
    }
    if (n > 0x7fffffff) return MPS_ERR_ARG;
    *n_out = int32_t(n);
    return MPS_OK;
}

int mps_scene_dambreak(const mps_scene_desc* d, int32_t cap, int8_t* typ, double* pos,
                       double* vel, double* nrm, int32_t* n_out) {
    int32_t n = 0;
    int rc = mps_scene_dambreak_count(d, &n);
    if (rc) return rc;
    if (n_out) *n_out = n;
    if (cap < n || !typ || !pos || !vel || !nrm) return MPS_ERR_ARG;
    const size_t N = size_t(cap);
    std::mt19937_64 jit(d->seed);
    Normal vn(d->vel_seed);
    const double l0 = d->l0, amp = d->jitter * l0;
    size_t id = 0;
    auto put = [&](int t, double x, double y, double z, double u, double v, double w, double a,
                   double b, double c) {
        typ[id] = int8_t(t);
        pos[id] = x + d->origin[0]; pos[N + id] = y + d->origin[1]; pos[2 * N + id] = z + d->origin[2];
        vel[id] = u; vel[N + id] = v; vel[2 * N + id] = w;
        nrm[id] = a; nrm[N + id] = b; nrm[2 * N + id] = c;
        ++id;
    };
    // fluid block, x fastest
    for (int k = 0; k < d->block[2]; ++k)
        for (int j = 0; j < d->block[1]; ++j)
            for (int i = 0; i < d->block[0]; ++i) {
                double x = (i + 0.5) * l0, y = (j + 0.5) * l0, z = (k + 0.5) * l0;
                x += (2.0 * u01(jit) - 1.0) * amp;
                y += (2.0 * u01(jit) - 1.0) * amp;
                z += (2.0 * u01(jit) - 1.0) * amp;
                double u = 0, v = 0, w = 0;
                if (d->vel_sigma > 0) {
                    u = d->vel_sigma * vn.next();
                    v = d->vel_sigma * vn.next();
                    w = d->vel_sigma * vn.next();
                }
                put(MPS_FLD, x, y, z, u, v, w, 0, 0, 0);
            }
    // walls: faces x=0, x=Lx, y=0, y=Ly, z=0, z=Lz
    for (int f = 0; f < 6; ++f) {
        if (!(d->wall_mask & (1 << f))) continue;
        int nn[3];
        face_points(*d, f, nn);
        const int axis = f / 2;
        const double plane = (f % 2) ? d->tank[axis] : 0.0;
        const double sgn = (f % 2) ? -1.0 : 1.0;
        const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
        for (int q = 0; q < nn[a2]; ++q)
            for (int p = 0; p < nn[a1]; ++p) {
                double c[3], nv[3] = {0, 0, 0};
                c[axis] = plane;
                c[a1] = (p + 0.5) * l0;
                c[a2] = (q + 0.5) * l0;
                nv[axis] = sgn;
                put(MPS_WLL, c[0], c[1], c[2], 0, 0, 0, nv[0], nv[1], nv[2]);
            }
    }
    return MPS_OK;
}

int mps_params_dambreak(const mps_scene_desc* d, double snd, double dt, double knm_vsc,
                        double g_z, int32_t precision, mps_params* p) {
    if (!valid(d) || !p) return MPS_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->pcl_dst = d->l0;
    for (int a = 0; a < 3; ++a) {
        p->min[a] = d->origin[a];
        p->max[a] = d->origin[a] + d->tank[a];
    }
    p->g[2] = g_z;
    p->knm_vsc = knm_vsc;
    // COL_RAT / DST_LMT_RAT: the reference reads them from MPS_physical.txt, which it does
    // not ship; these are the values used throughout this project
    p->col_rat = 0.2;
    p->dst_lmt_rat = 0.9;
    p->rho = 1000.0;  // Dns_FLD, const.cuh:38
    p->snd = snd;
    p->dt = dt;
    // SetPara: umax = sqrt(2|g|H), Pmax = rho g H with H the fluid extent (max - min of the
    // particle centres) along gravity (kernel.cu:399-411, taken along z here)
    const double H = d->block[2] > 0 ? (d->block[2] - 1) * d->l0 : 0.0;
    p->umax = std::sqrt(2.0 * std::fabs(g_z) * H);
    p->pmax = p->rho * std::fabs(g_z) * H;
    p->precision = precision;
    return MPS_OK;
}

}  // extern "C"
