// oracle_scene.cpp -- dam-break scenes and their parameters for the oracle side
// (TEST INFRASTRUCTURE, not the product).
//
// bench.py's reference arm and the CPU baselines build their input here, so that timing the
// reference's loops never maps the product library. The definition is the one the product's
// generator (mps_scene_dambreak / mps_params_dambreak) documents, restated on its own:
//   * fluid: block[0] x block[1] x block[2] particles at ((i+1/2) l0, (j+1/2) l0, (k+1/2) l0),
//     i fastest, each coordinate moved by (2u - 1) * jitter * l0 with u = (g() >> 11) * 2^-53
//     drawn from std::mt19937_64(seed) in the order x, y, z; with vel_sigma > 0 each fluid
//     particle then takes three N(0, vel_sigma) velocities from a second mt19937_64(vel_seed),
//     Box-Muller in pairs (radius * cos first, radius * sin kept for the next draw);
//   * walls: for each face f = 0..5 in wall_mask (x = 0, x = Lx, y = 0, y = Ly, z = 0, z = Lz)
//     one layer on the face plane at ((p+1/2) l0, (q+1/2) l0) in its two other axes (the
//     lower-numbered one fastest), round(L / l0) points per axis, with the inward unit normal;
//   * every position is offset by `origin`.
// SetPara's explicit values (kernel.cu:396-415, taken along gravity on z): umax =
// sqrt(2 |g| H), Pmax = rho |g| H, H = (block[2] - 1) l0; COL_RAT 0.2, DST_LMT_RAT 0.9 (the
// reference reads both from an MPS_physical.txt it does not ship); rho = 1000 (const.cuh:38).
// tests/test_oracle_scene.py checks that both generators give the same bytes.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>

#include "mps_oracle.h"

namespace {

constexpr double kTwoPow53 = 9007199254740992.0;

double uniform53(std::mt19937_64& rng) { return double(rng() >> 11) / kTwoPow53; }

class GaussPairs {
   public:
    explicit GaussPairs(uint64_t seed) : rng_(seed) {}
    double draw() {
        if (pending_) {
            pending_ = false;
            return second_;
        }
        double a = uniform53(rng_);
        const double b = uniform53(rng_);
        if (a <= 0.0) a = 1.0 / kTwoPow53;
        const double radius = std::sqrt(-2.0 * std::log(a));
        const double angle = 6.283185307179586 * b;
        second_ = radius * std::sin(angle);
        pending_ = true;
        return radius * std::cos(angle);
    }

   private:
    std::mt19937_64 rng_;
    bool pending_ = false;
    double second_ = 0.0;
};

bool desc_ok(const oracle_scene_desc* d) {
    if (d == nullptr || !(d->l0 > 0)) return false;
    for (int a = 0; a < 3; ++a)
        if (!(d->tank[a] > 0) || d->block[a] < 0) return false;
    return true;
}

// points of face f per axis (n[3]) and their number
long long face_layout(const oracle_scene_desc& d, int f, long long n[3]) {
    for (int a = 0; a < 3; ++a) n[a] = std::lround(d.tank[a] / d.l0);
    const int normal_axis = f / 2;
    long long total = 1;
    for (int a = 0; a < 3; ++a)
        if (a != normal_axis) total *= n[a];
    return total;
}

long long scene_size(const oracle_scene_desc& d) {
    long long total = (long long)d.block[0] * d.block[1] * d.block[2];
    for (int f = 0; f < 6; ++f) {
        if ((d.wall_mask >> f) & 1) {
            long long n[3];
            total += face_layout(d, f, n);
        }
    }
    return total;
}

}  // namespace

extern "C" {

int oracle_scene_dambreak_count(const oracle_scene_desc* d, int32_t* n_out) {
    if (!desc_ok(d) || n_out == nullptr) return 1;
    const long long n = scene_size(*d);
    if (n > 0x7fffffffLL) return 1;
    *n_out = int32_t(n);
    return 0;
}

int oracle_scene_dambreak(const oracle_scene_desc* d, int32_t cap, int8_t* typ, double* pos,
                          double* vel, double* nrm) {
    int32_t n = 0;
    if (oracle_scene_dambreak_count(d, &n) != 0 || cap < n || !typ || !pos || !vel || !nrm)
        return 1;
    const size_t stride = size_t(cap);
    std::mt19937_64 jitter_rng(d->seed);
    GaussPairs gauss(d->vel_seed);
    const double l0 = d->l0, amplitude = d->jitter * d->l0;
    size_t at = 0;
    auto emit = [&](int8_t t, const double x[3], const double u[3], const double nv[3]) {
        typ[at] = t;
        for (int a = 0; a < 3; ++a) {
            pos[a * stride + at] = x[a] + d->origin[a];
            vel[a * stride + at] = u[a];
            nrm[a * stride + at] = nv[a];
        }
        ++at;
    };
    const double zero[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < d->block[2]; ++k)
        for (int j = 0; j < d->block[1]; ++j)
            for (int i = 0; i < d->block[0]; ++i) {
                const int idx[3] = {i, j, k};
                double x[3], u[3] = {0.0, 0.0, 0.0};
                for (int a = 0; a < 3; ++a) x[a] = (idx[a] + 0.5) * l0;
                for (int a = 0; a < 3; ++a) x[a] += (2.0 * uniform53(jitter_rng) - 1.0) * amplitude;
                if (d->vel_sigma > 0)
                    for (int a = 0; a < 3; ++a) u[a] = d->vel_sigma * gauss.draw();
                emit(0 /* FLD */, x, u, zero);
            }
    for (int f = 0; f < 6; ++f) {
        if (!((d->wall_mask >> f) & 1)) continue;
        long long npt[3];
        face_layout(*d, f, npt);
        const int na = f / 2;
        const bool far_side = (f & 1) != 0;
        const int fast = na == 0 ? 1 : 0, slow = na == 2 ? 1 : 2;
        double nv[3] = {0.0, 0.0, 0.0};
        nv[na] = far_side ? -1.0 : 1.0;
        for (long long q = 0; q < npt[slow]; ++q)
            for (long long p = 0; p < npt[fast]; ++p) {
                double x[3];
                x[na] = far_side ? d->tank[na] : 0.0;
                x[fast] = (p + 0.5) * l0;
                x[slow] = (q + 0.5) * l0;
                emit(1 /* WLL */, x, zero, nv);
            }
    }
    return 0;
}

int oracle_params_dambreak(const oracle_scene_desc* d, double snd, double dt, double knm_vsc,
                           double g_z, int32_t precision, oracle_params* p) {
    if (!desc_ok(d) || p == nullptr) return 1;
    std::memset(p, 0, sizeof(*p));
    p->pcl_dst = d->l0;
    for (int a = 0; a < 3; ++a) {
        p->min[a] = d->origin[a];
        p->max[a] = d->origin[a] + d->tank[a];
    }
    p->g[2] = g_z;
    p->knm_vsc = knm_vsc;
    p->col_rat = 0.2;
    p->dst_lmt_rat = 0.9;
    p->rho = 1000.0;
    p->snd = snd;
    p->dt = dt;
    const double height = d->block[2] > 0 ? (d->block[2] - 1) * d->l0 : 0.0;
    p->umax = std::sqrt(2.0 * std::fabs(g_z) * height);
    p->pmax = p->rho * std::fabs(g_z) * height;
    p->precision = precision;
    return 0;
}

}  // extern "C"
