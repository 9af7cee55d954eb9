// mps_types.h -- host/device data layout of the B200 MPS solver.
//
// Particle state lives in HBM as arrays of 4-wide vectors (16 B per float particle,
// 32 B per double particle). Fluid is sorted by the reference's bucket, then by fine cell
// inside it (a third of a bucket per axis), ascending particle id inside a fine cell, so
// that a neighbour walk reads only the fine cells its radius reaches. Walls are static and sorted
// by the reference's bucket order ib = iz*nBxy + iy*nBx + ix (kernel.cu:521-524), ascending
// id inside a bucket; mirrors are a compact list sorted by (bucket, slot id) instead of
// the reference's NumMRR slots per particle (kernel.cu:96-103).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define MPS_HD __host__ __device__ __forceinline__
#else
#define MPS_HD inline
#endif

namespace mps {

constexpr int kGST = -1, kFLD = 0, kWLL = 1, kOBJ = 2, kOBJ2 = 3, kMRR = 4;
constexpr int kEDGE = 1;
constexpr int kNumMRR = 10;  // const.cuh:50

template <class R> struct alignas(4 * sizeof(R)) V4 {
    R x, y, z, w;
};

// Per-scene constants, derived on the host exactly as AlcBkt/SetPara do (kernel.cu:307-415).
template <class R, class RN> struct SceneDev {
    R minc[3];        // padded domain minimum (kernel.cu:26-28)
    R dbinv, db;      // bucket width 3.1 l0 and its inverse (kernel.cu:313-315)
    int nbx, nby, nbz, nbxy;
    int cbase;        // first global bucket of this scene
    int pbase;        // first global particle id of this scene
    int pcount;       // particles of this scene
    // fluid lists use fine cells, a third of a bucket per axis and nested in the buckets,
    // numbered fbase + 27 * bucket + 9 sz + 3 sy + sx (sub-cell s = int(3 t) + 3 - 3 i,
    // t as for the bucket index i)
    int fbase, pad1, pad2;
    float hf, ihf;    // fine cell width (bucket width / 3) and its inverse
    R r, r2, r_le;    // Laplacian radius; r_le = largest t with sqrt(t) <= r
    R rp, rp2, rp_lt; // gradient radius; rp_lt = largest t with sqrt(t) < rp
    R rlim2, rlimw2;  // collision radii (kernel.cu:370-371, 1184-1185)
    R list_thr;       // d2 bound of the neighbour lists shared by ChkCol/MkPrs/PrsGrdTrm
    R edge_r2;        // Surface_Edge radius^2 (kernel.cu:558)
    R wall_dist0;     // 10 r (kernel.cu:940)
    R two_l0, kn;     // 2 l0; KNM_VSC / n0 (kernel.cu:1113)
    R g[3];
    R dt, umax;
    R lo[3], hi[3];   // ChkPcl box (kernel.cu:484-486)
    R colfac;         // COL * mj / (mi + mj) (kernel.cu:1215)
    R invro, a3;      // -1/rho, 3/n0_grad (kernel.cu:1659, 1665)
    R invn0g;         // 1/n0_grad (kernel.cu:1443, the corrected-gradient variant)
    // (radius + margin)^2 used to skip bucket rows: r, rp, rlim, 0.45 l0, max(rlim, rp)
    R skip_r, skip_rp, skip_rl, skip_rw, skip_rc;
    RN n0g, prs_coef, pmax, rho;          // number density / EOS in RN (kernel.cu:1388-1406)
    RN rp_n;
};

// Prescribed rigid motion of one moving-wall type (OBJ or OBJ2), in double: a wall particle
// set moving at x0 with normal n0 is at c + t + q (x0 - c) with normal q n0 and velocity
// v + w x (q (x0 - c)), where q and t accumulate one step's rotation qs and translation vdt.
struct WallMotion {
    double qs[9];   // rotation of one step, row-major
    double q[9];    // rotation since the motion was set
    double c[3];    // centre of rotation when the motion was set
    double t[3];    // translation since the motion was set
    double vdt[3];  // translation of one step
    double w[3];    // angular velocity vector
    double v[3];    // translation velocity
    int type;       // particle type that moves (kOBJ or kOBJ2), 0 when off
    int pad;
};

struct DevCounters {
    int mirror_raw;       // entries appended to the raw mirror list
    int err_mirror_slot;  // corner mirror without a free slot (kernel.cu:868-874)
    int err_capacity;     // raw mirror list full
    int err_cell;         // bucket index clamped into the grid
    int err_nan;          // non-finite position met in a bucket build
    int n_m1, n_m2;       // alive mirrors after the latest generations
    int deleted;          // particles deleted by ChkPcl (cumulative)
    int scan_ticket;      // blocks of the running fine-cell scan that finished (0 between)
    int stage_blocks;     // blocks of a staged pass that walked shared memory (diagnostics)
    int unstaged_blocks;  // ... and those whose neighbourhood did not fit (diagnostics)
    int pad[5];
    // diagnostics: fluid candidates tested by VscTrm's walk and by the list build of
    // ChkCol/MkPrs, and the entries of those lists
    unsigned long long work[3];
};

}  // namespace mps
