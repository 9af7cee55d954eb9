// mps_device.cuh -- per-particle physics of the explicit MPS step, as device functions.
//
// Every function here is shared by the fused step kernels and by the one-method-per-launch
// kernels behind mps_phase(), so both paths round identically. Arithmetic follows one
// fixed form (the build uses -fmad=false; each fused multiply-add is an explicit
// __fma_rn), neighbour buckets are visited z, y, x ascending and particles inside a bucket
// in ascending id, so a result depends only on its inputs.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "mps_types.h"

namespace mps {

__device__ __forceinline__ float fmaR(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaR(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float sqrtR(float a) { return sqrtf(a); }
__device__ __forceinline__ double sqrtR(double a) { return sqrt(a); }

template <class R> __device__ __forceinline__ R dot3(R ax, R ay, R az, R bx, R by, R bz) {
    return fmaR(az, bz, fmaR(ay, by, ax * bx));
}
// WEI_grad(dst, re), const.cuh:46
template <class R> __device__ __forceinline__ R wei_grad(R d, R re) { return (re / d) - (d / re); }

template <class R> __device__ __forceinline__ V4<R> ldv(const V4<R>* p) {
    return __ldg(reinterpret_cast<const V4<R>*>(p));
}
__device__ __forceinline__ V4<float> ldg4(const V4<float>* p) {
    float4 v = __ldg(reinterpret_cast<const float4*>(p));
    return V4<float>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ldg4(const V4<double>* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return V4<double>{a.x, a.y, b.x, b.y};
}

// scene of a global particle id (scenes are stored in ascending pbase)
template <class R, class RN>
__device__ __forceinline__ int scene_of(const SceneDev<R, RN>* sc, int nscene, int pid) {
    int lo = 0, hi = nscene - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&sc[mid].pbase) <= pid) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Bucket coordinates, kernel.cu:521-524. Returns false if the index left the grid (then
// it is clamped to the interior so that the 27-bucket walk stays inside the grid).
template <class R, class RN>
__device__ __forceinline__ bool cell_of(const SceneDev<R, RN>& sc, R x, R y, R z, int& ix,
                                        int& iy, int& iz) {
    ix = int((x - sc.minc[0]) * sc.dbinv) + 1;
    iy = int((y - sc.minc[1]) * sc.dbinv) + 1;
    iz = int((z - sc.minc[2]) * sc.dbinv) + 1;
    bool ok = ix >= 1 && ix <= sc.nbx - 2 && iy >= 1 && iy <= sc.nby - 2 && iz >= 1 &&
              iz <= sc.nbz - 2;
    if (!ok) {
        ix = min(max(ix, 1), sc.nbx - 2);
        iy = min(max(iy, 1), sc.nby - 2);
        iz = min(max(iz, 1), sc.nbz - 2);
    }
    return ok;
}

// Position of a particle inside its bucket, used to skip bucket rows that cannot hold a
// neighbour inside the radius. Skipping never reorders the neighbours that remain.
template <class R> struct RowCtx {
    int ix, iy, iz;
    R dxl, dxh, dyl, dyh, dzl, dzh;
    float rx, ry, rz;  // position relative to the grid minimum (fine-row geometry)
};

template <class R, class RN>
__device__ __forceinline__ RowCtx<R> row_ctx(const SceneDev<R, RN>& sc, R x, R y, R z, int ix,
                                             int iy, int iz) {
    RowCtx<R> c;
    c.ix = ix; c.iy = iy; c.iz = iz;
    R xl = sc.minc[0] + R(ix - 1) * sc.db;
    R yl = sc.minc[1] + R(iy - 1) * sc.db;
    R zl = sc.minc[2] + R(iz - 1) * sc.db;
    c.dxl = x - xl; c.dxh = (xl + sc.db) - x;
    c.dyl = y - yl; c.dyh = (yl + sc.db) - y;
    c.dzl = z - zl; c.dzh = (zl + sc.db) - z;
    c.rx = float(x - sc.minc[0]);
    c.ry = float(y - sc.minc[1]);
    c.rz = float(z - sc.minc[2]);
    return c;
}

// Fine cell of a fluid particle: a third of its bucket per axis. t = (x - min) * dbinv is
// the bucket coordinate of kernel.cu:521-524 and the fine coordinate is fx = int(3 t) + 3;
// for t >= 0 rounding keeps int(3 t) in [3 int(t), 3 int(t) + 2], so the fine cell lies
// inside the bucket. The clamp repeats cell_of's for positions outside the grid. Fine cells
// are numbered bucket-major (27 per bucket, z, y, x inside it), so that consecutive slots
// stay within one bucket.
template <class R, class RN>
__device__ __forceinline__ int fine_cell(const SceneDev<R, RN>& sc, R x, R y, R z, bool& ok) {
    const R tx = (x - sc.minc[0]) * sc.dbinv, ty = (y - sc.minc[1]) * sc.dbinv,
            tz = (z - sc.minc[2]) * sc.dbinv;
    int ix = int(tx) + 1, iy = int(ty) + 1, iz = int(tz) + 1;
    ok = ix >= 1 && ix <= sc.nbx - 2 && iy >= 1 && iy <= sc.nby - 2 && iz >= 1 && iz <= sc.nbz - 2;
    ix = min(max(ix, 1), sc.nbx - 2);
    iy = min(max(iy, 1), sc.nby - 2);
    iz = min(max(iz, 1), sc.nbz - 2);
    const int sx = min(max(int(R(3) * tx) + 3, 3 * ix), 3 * ix + 2) - 3 * ix;
    const int sy = min(max(int(R(3) * ty) + 3, 3 * iy), 3 * iy + 2) - 3 * iy;
    const int sz = min(max(int(R(3) * tz) + 3, 3 * iz), 3 * iz + 2) - 3 * iz;
    return sc.fbase + 27 * (iz * sc.nbxy + iy * sc.nbx + ix) + 9 * sz + 3 * sy + sx;
}

// first / last fine index of the 9 around the bucket (f0 = 3 i - 3) whose cells reach
// coordinate v; v * ihf + 3 is the fine coordinate
__device__ __forceinline__ int fine_at(float v, float ihf, int f0) {
    return int(fminf(fmaxf(fmaf(v, ihf, 3.0f), float(f0)), float(f0 + 8)));
}
// distance from v to fine cell f along one axis
__device__ __forceinline__ float fine_gap(float v, int f, float hf) {
    const float lo = float(f - 3) * hf;
    return fmaxf(fmaxf(lo - v, v - (lo + hf)), 0.0f);
}

// A fluid slot index kept in the w component of a position (the row-ordered copy posf)
__device__ __forceinline__ float slot_w(int s, float) { return __int_as_float(s); }
__device__ __forceinline__ double slot_w(int s, double) { return double(s); }
__device__ __forceinline__ int w_slot(float w) { return __float_as_int(w); }
__device__ __forceinline__ int w_slot(double w) { return int(w); }

// Row-major number of bucket-major fine cell c (fz * 9 nbxy + fy * 3 nbx + fx): the order
// of the copy posf, in which one fine row across the 27 buckets is one contiguous range.
template <class R, class RN>
__device__ __forceinline__ int fine_rowmajor(const SceneDev<R, RN>& sc, int c) {
    const int l = c - sc.fbase, b = l / 27, sub = l - 27 * b;
    const int bz = b / sc.nbxy, by = (b - bz * sc.nbxy) / sc.nbx, bx = b - bz * sc.nbxy - by * sc.nbx;
    const int fz = 3 * bz + sub / 9, fy = 3 * by + (sub / 3) % 3, fx = 3 * bx + sub % 3;
    return sc.fbase + fz * (9 * sc.nbxy) + fy * (3 * sc.nbx) + fx;
}

// The fine rows of the fluid walk below: g(fz, fy, xl, xh) for every fine row (fz, fy) within sqrt(B),
// z then y ascending, with the fine cells [xl, xh] of the row it reaches. Every step is
// monotone in the particle's coordinates (IEEE arithmetic, clamps, truncation), which the
// staged walk relies on to bound the rows of a whole block from the box around its
// particles (stage_fluid).
template <class R, class RN, class G>
__device__ __forceinline__ void for_fluid_rows(const SceneDev<R, RN>& sc, const RowCtx<R>& c, R B,
                                               G&& g) {
    const float b = float(B), hf = sc.hf, ih = sc.ihf;
    const float s = sqrtf(b);
    const int fx0 = 3 * c.ix - 3, fy0 = 3 * c.iy - 3, fz0 = 3 * c.iz - 3;
    const int zl = fine_at(c.rz - s, ih, fz0), zh = fine_at(c.rz + s, ih, fz0);
    for (int fz = zl; fz <= zh; ++fz) {
        const float gz = fine_gap(c.rz, fz, hf);
        const float bz = fmaxf(b - gz * gz, 0.0f), sy = sqrtf(bz);
        const int yl = fine_at(c.ry - sy, ih, fy0), yh = fine_at(c.ry + sy, ih, fy0);
        for (int fy = yl; fy <= yh; ++fy) {
            const float gy = fine_gap(c.ry, fy, hf);
            const float sx = sqrtf(fmaxf(bz - gy * gy, 0.0f));
            g(fz, fy, fine_at(c.rx - sx, ih, fx0), fine_at(c.rx + sx, ih, fx0));
        }
    }
}

// Visit the fluid of the 27 buckets around c in fine cells, z, y, x ascending, ascending
// particle id inside a fine cell, through the row-ordered copy posf (start table csr):
// f(lo, hi) for the range of posf of every fine row's cells within sqrt(B) of the particle.
// `B` is (radius + margin)^2, the margin (1e-3 of a bucket) covering the float geometry. The
// neighbours inside the radius, and their order, are those of a walk over every fine cell
// of the 27 buckets.
template <class R, class RN, class F>
__device__ __forceinline__ void for_fluid_ranges(const SceneDev<R, RN>& sc,
                                                 const int* __restrict__ csr, const RowCtx<R>& c,
                                                 R B, F&& f) {
    const int nfx = 3 * sc.nbx, nfxy = 9 * sc.nbxy;
    for_fluid_rows(sc, c, B, [&](int fz, int fy, int xl, int xh) {
        const int row = sc.fbase + fz * nfxy + fy * nfx;
        f(__ldg(csr + row + xl), __ldg(csr + row + xh + 1));
    });
}

template <class R, class RN, class F>
__device__ __forceinline__ void for_fluid(const SceneDev<R, RN>& sc, const int* __restrict__ csr,
                                          const V4<R>* __restrict__ posf, const RowCtx<R>& c, R B,
                                          F&& f) {
    for_fluid_ranges(sc, csr, c, B, [&](int lo, int hi) {
        for (int k = lo; k < hi; ++k) {
            const V4<R> q = ldg4(posf + k);
            f(w_slot(q.w), q);
        }
    });
}

// Visit the 27 buckets around c (z, y, x ascending); a row of three x-adjacent buckets is
// one contiguous range of the sorted arrays. The row loops stay rolled: the visit bodies
// (collision, density, gradient, mirror generation) are long, and nine copies of each
// overflow the instruction cache. `B` is (radius + margin)^2: a row or an end
// bucket whose nearest point lies farther than that is not visited.
template <class R, class RN, class F>
__device__ __forceinline__ void for_rows(const SceneDev<R, RN>& sc, const int* __restrict__ cs,
                                         const RowCtx<R>& c, R B, F&& f) {
#pragma unroll 1
    for (int dz = -1; dz <= 1; ++dz) {
        R ddz = dz < 0 ? c.dzl : (dz > 0 ? c.dzh : R(0));
#pragma unroll 1
        for (int dy = -1; dy <= 1; ++dy) {
            R ddy = dy < 0 ? c.dyl : (dy > 0 ? c.dyh : R(0));
            R dyz2 = ddy * ddy + ddz * ddz;
            if (dyz2 > B) continue;
            int jl = (dyz2 + c.dxl * c.dxl <= B) ? c.ix - 1 : c.ix;
            int jh = (dyz2 + c.dxh * c.dxh <= B) ? c.ix + 1 : c.ix;
            int row = sc.cbase + (c.iz + dz) * sc.nbxy + (c.iy + dy) * sc.nbx;
            int lo = __ldg(cs + row + jl), hi = __ldg(cs + row + jh + 1);
            for (int j = lo; j < hi; ++j) f(j);
        }
    }
}

// for_rows, handing each (trimmed) row range [lo, hi) to f(lo, hi) in visiting order
template <class R, class RN, class F>
__device__ __forceinline__ void for_rows_ranges(const SceneDev<R, RN>& sc,
                                                const int* __restrict__ cs, const RowCtx<R>& c,
                                                R B, F&& f) {
#pragma unroll 1
    for (int dz = -1; dz <= 1; ++dz) {
        R ddz = dz < 0 ? c.dzl : (dz > 0 ? c.dzh : R(0));
#pragma unroll 1
        for (int dy = -1; dy <= 1; ++dy) {
            R ddy = dy < 0 ? c.dyl : (dy > 0 ? c.dyh : R(0));
            R dyz2 = ddy * ddy + ddz * ddz;
            if (dyz2 > B) continue;
            int jl = (dyz2 + c.dxl * c.dxl <= B) ? c.ix - 1 : c.ix;
            int jh = (dyz2 + c.dxh * c.dxh <= B) ? c.ix + 1 : c.ix;
            int row = sc.cbase + (c.iz + dz) * sc.nbxy + (c.iy + dy) * sc.nbx;
            f(__ldg(cs + row + jl), __ldg(cs + row + jh + 1));
        }
    }
}

// ---- views ------------------------------------------------------------------------------
template <class R> struct WallView {
    const int* cs;
    const V4<R>* pos;
    const V4<R>* nrm;
    const V4<R>* vel;
    const int8_t* wse;
    const int8_t* typ;
};
template <class R> struct MirrorView {
    const int* cs;
    const V4<R>* pos;  // w = PrsM
    const int* slot;
};
template <class R> struct MirrorSink {
    V4<R>* pos;
    int* slot;
    int cap;
    // recorded rollouts only: per raw mirror n * sqrt(2 / |n|) of its reflection plane's
    // normal n, so that d(mirror)/d(owner) = I - nrm nrm^T
    V4<R>* nrm;
};

// ---- VscTrm sum (kernel.cu:1037-1107) ----------------------------------------------------
// mirror part: VelM = 0 (kernel.cu:834-836)
template <class R, class RN>
__device__ __forceinline__ void visc_sum_mirrors(const SceneDev<R, RN>& sc, const RowCtx<R>& c, R x,
                                                 R y, R z, R ux, R uy, R uz,
                                                 const MirrorView<R>& m, R B, R& sx, R& sy, R& sz,
                                                 int& cm) {
    for_rows(sc, m.cs, c, B, [&](int k) {
        V4<R> q = ldg4(m.pos + k);
        R dx = q.x - x, dy = q.y - y, dz = q.z - z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 <= sc.r_le) {
            R d = sqrtR(d2);
            R w = sc.two_l0 / (d2 * d);
            sx = fmaR(R(0) - ux, w, sx);
            sy = fmaR(R(0) - uy, w, sy);
            sz = fmaR(R(0) - uz, w, sz);
            ++cm;
        }
    });
}

template <class R, class RN>
__device__ __forceinline__ void visc_sum(const SceneDev<R, RN>& sc, const RowCtx<R>& c, int s,
                                         R x, R y, R z, R ux, R uy, R uz,
                                         const int* __restrict__ csr,
                                         const V4<R>* __restrict__ posf,
                                         const V4<R>* __restrict__ vel, const MirrorView<R>& m,
                                         R B, R& sx, R& sy, R& sz, int& cf, int& cm) {
    for_fluid(sc, csr, posf, c, B, [&](int j, const V4<R>& q) {
        if (j == s) return;
        R dx = q.x - x, dy = q.y - y, dz = q.z - z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 <= sc.r_le) {  // dist <= r
            V4<R> u = ldg4(vel + j);
            R d = sqrtR(d2);
            R w = sc.two_l0 / (d2 * d);
            sx = fmaR(u.x - ux, w, sx);
            sy = fmaR(u.y - uy, w, sy);
            sz = fmaR(u.z - uz, w, sz);
            ++cf;
        }
    });
    visc_sum_mirrors(sc, c, x, y, z, ux, uy, uz, m, B, sx, sy, sz, cm);
}

// ---- ChkPcl (kernel.cu:481-513); returns false when the particle is deleted --------------
template <class R, class RN>
__device__ __forceinline__ bool chkpcl(const SceneDev<R, RN>& sc, R x, R y, R z, R& ux, R& uy,
                                       R& uz) {
    if (x < sc.hi[0] && x > sc.lo[0] && y < sc.hi[1] && y > sc.lo[1] && z < sc.hi[2] &&
        z > sc.lo[2]) {
        R u = sqrtR(dot3(ux, uy, uz, ux, uy, uz));
        if (u > sc.umax) {
            R f = sc.umax / u;
            ux *= f; uy *= f; uz *= f;
        }
        return true;
    }
    return false;
}

// ---- ChkCol (kernel.cu:1193-1275) and MkPrs (kernel.cu:1328-1386) sums ------------------
template <class R>
__device__ __forceinline__ void col_hit(R colfac, R ux, R uy, R uz, R jx, R jy, R jz, R dx, R dy,
                                        R dz, R d2, R& wx, R& wy, R& wz) {
    R f = dot3(ux - jx, uy - jy, uz - jz, dx, dy, dz);
    if (f > R(0)) {
        f = f * (colfac / d2);
        wx = fmaR(-dx, f, wx);
        wy = fmaR(-dy, f, wy);
        wz = fmaR(-dz, f, wz);
    }
}

template <class R, class RN>
__device__ __forceinline__ void dens_add_v(R rp, RN rp_n, R d2, RN& ni) {
    if (sizeof(RN) == sizeof(R)) {
        R d = sqrtR(d2);
        ni += RN(wei_grad(d, rp));
    } else {
        RN d = sqrtR(RN(d2));
        ni += wei_grad(d, rp_n);
    }
}
template <class R, class RN>
__device__ __forceinline__ void dens_add(const SceneDev<R, RN>& sc, R d2, RN& ni) {
    dens_add_v(sc.rp, sc.rp_n, d2, ni);
}

// wall (collision only) and mirror parts, visited after the fluid neighbours
template <class R, class RN, bool COL, bool DENS>
__device__ __forceinline__ void col_dens_walls_mirrors(const SceneDev<R, RN>& sc, const RowCtx<R>& c,
                                                       R x, R y, R z, R ux, R uy, R uz,
                                                       const WallView<R>& wl,
                                                       const MirrorView<R>& m, bool skip, R& wx,
                                                       R& wy, R& wz, RN& ni, int* cnt,
                                                       bool walls = true, bool mirrors = true) {
    const R inf = R(INFINITY);
    const R Bf = !skip ? inf : (COL && DENS ? sc.skip_rc : (DENS ? sc.skip_rp : sc.skip_rl));
    if (COL && walls) {
        for_rows(sc, wl.cs, c, skip ? sc.skip_rw : inf, [&](int j) {
            V4<R> q = ldg4(wl.pos + j);
            R dx = q.x - x, dy = q.y - y, dz = q.z - z;
            R d2 = dot3(dx, dy, dz, dx, dy, dz);
            if (d2 < sc.rlimw2) {
                V4<R> u = ldg4(wl.vel + j);
                col_hit(sc.colfac, ux, uy, uz, u.x, u.y, u.z, dx, dy, dz, d2, wx, wy, wz);
                ++cnt[1];
            }
        });
    }
    if (!mirrors) return;
    for_rows(sc, m.cs, c, Bf, [&](int k) {
        V4<R> q = ldg4(m.pos + k);
        R dx = q.x - x, dy = q.y - y, dz = q.z - z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (COL && d2 < sc.rlim2) {
            col_hit(sc.colfac, ux, uy, uz, R(0), R(0), R(0), dx, dy, dz, d2, wx, wy, wz);
            ++cnt[2];
        }
        if (DENS && d2 <= sc.rp_lt) {
            dens_add(sc, d2, ni);
            ++cnt[4];
        }
    });
}

template <class R, class RN, bool COL, bool DENS>
__device__ __forceinline__ void col_dens_sum(const SceneDev<R, RN>& sc, const RowCtx<R>& c, int s,
                                             R x, R y, R z, R ux, R uy, R uz,
                                             const int* __restrict__ csr,
                                             const V4<R>* __restrict__ posf,
                                             const V4<R>* __restrict__ vel,
                                             const WallView<R>& wl, const MirrorView<R>& m,
                                             bool skip, R& wx, R& wy, R& wz, RN& ni, int* cnt) {
    const R inf = R(INFINITY);
    const R Bf = !skip ? inf : (COL && DENS ? sc.skip_rc : (DENS ? sc.skip_rp : sc.skip_rl));
    for_fluid(sc, csr, posf, c, Bf, [&](int j, const V4<R>& q) {
        if (j == s) return;
        R dx = q.x - x, dy = q.y - y, dz = q.z - z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (COL && d2 < sc.rlim2) {
            V4<R> u = ldg4(vel + j);
            col_hit(sc.colfac, ux, uy, uz, u.x, u.y, u.z, dx, dy, dz, d2, wx, wy, wz);
            ++cnt[0];
        }
        if (DENS && d2 <= sc.rp_lt) {  // dist < rp
            dens_add(sc, d2, ni);
            ++cnt[3];
        }
    });
    col_dens_walls_mirrors<R, RN, COL, DENS>(sc, c, x, y, z, ux, uy, uz, wl, m, skip, wx, wy, wz,
                                             ni, cnt);
}

// explicit equation of state with clamps, kernel.cu:1388-1406
template <class R, class RN>
__device__ __forceinline__ R eos(const SceneDev<R, RN>& sc, RN ni) {
    RN p = RN(ni > sc.n0g ? 1 : 0) * (ni - sc.n0g) * sc.prs_coef * sc.rho;
    if (p <= sc.pmax && p >= RN(0)) {
    } else {
        p = (p > sc.pmax) ? sc.pmax : RN(0);
    }
    return R(p);
}

// ---- PrsGrdTrm (kernel.cu:1678-1791) ----------------------------------------------------
// The sums over the neighbours inside rp, w = WEI_grad(d, rp) / d^2 and r = x_j - x_i.
// GradPlain is the compiled variant: b = sum w (P_j - P_min) r (kernel.cu:1728-1735).
// GradCorr is the corrected-matrix #if 0 variant (kernel.cu:1535-1548): also the moment
// matrix M = sum w r r^T, entry (a, b) accumulated as (w r_a) r_b, all nine kept apart.
template <class R> struct GradPlain {
    R sx = R(0), sy = R(0), sz = R(0);
    __device__ __forceinline__ void add(R w, R pd, R dx, R dy, R dz) {
        const R pw = pd * w;
        sx = fmaR(pw, dx, sx);
        sy = fmaR(pw, dy, sy);
        sz = fmaR(pw, dz, sz);
    }
};
template <class R> struct GradCorr {
    R m0 = R(0), m1 = R(0), m2 = R(0), m3 = R(0), m4 = R(0), m5 = R(0), m6 = R(0), m7 = R(0),
      m8 = R(0);
    R b0 = R(0), b1 = R(0), b2 = R(0);
    __device__ __forceinline__ void add(R w, R pd, R dx, R dy, R dz) {
        const R wx = w * dx, wy = w * dy, wz = w * dz;
        m0 = fmaR(wx, dx, m0); m1 = fmaR(wx, dy, m1); m2 = fmaR(wx, dz, m2);
        m3 = fmaR(wy, dx, m3); m4 = fmaR(wy, dy, m4); m5 = fmaR(wy, dz, m5);
        m6 = fmaR(wz, dx, m6); m7 = fmaR(wz, dy, m7); m8 = fmaR(wz, dz, m8);
        const R wp = w * pd;
        b0 = fmaR(wp, dx, b0);
        b1 = fmaR(wp, dy, b1);
        b2 = fmaR(wp, dz, b2);
    }
};

// acceleration of the compiled variant: -1/rho * b * 3/n0_grad (kernel.cu:1788-1790)
template <class R, class RN>
__device__ __forceinline__ bool grad_acc(const SceneDev<R, RN>& sc, const GradPlain<R>& g, R& ax,
                                         R& ay, R& az) {
    ax = (sc.invro * g.sx) * sc.a3;
    ay = (sc.invro * g.sy) * sc.a3;
    az = (sc.invro * g.sz) * sc.a3;
    return true;
}
// of the corrected variant: M and b scaled by 1/n0_grad, M inverted through its adjugate and
// determinant, a = -1/rho M^-1 b (kernel.cu:1608-1642). False when all nine entries of M are
// zero: the reference then returns without writing d_Acc (kernel.cu:1620).
template <class R, class RN>
__device__ __forceinline__ bool grad_acc(const SceneDev<R, RN>& sc, const GradCorr<R>& g, R& ax,
                                         R& ay, R& az) {
    const R k = sc.invn0g;
    const R m0 = k * g.m0, m1 = k * g.m1, m2 = k * g.m2, m3 = k * g.m3, m4 = k * g.m4,
            m5 = k * g.m5, m6 = k * g.m6, m7 = k * g.m7, m8 = k * g.m8;
    if (m0 == R(0) && m1 == R(0) && m2 == R(0) && m3 == R(0) && m4 == R(0) && m5 == R(0) &&
        m6 == R(0) && m7 == R(0) && m8 == R(0))
        return false;
    const R det = R(1) / ((m0 * m4 * m8 + m1 * m5 * m6 + m2 * m3 * m7) -
                          (m2 * m4 * m6 + m0 * m5 * m7 + m1 * m3 * m8));
    const R l0 = det * (m4 * m8 - m5 * m7), l1 = det * -(m1 * m8 - m2 * m7),
            l2 = det * (m1 * m5 - m2 * m4);
    const R l3 = det * -(m3 * m8 - m5 * m6), l4 = det * (m0 * m8 - m2 * m6),
            l5 = det * -(m0 * m5 - m2 * m3);
    const R l6 = det * (m3 * m7 - m4 * m6), l7 = det * -(m0 * m7 - m1 * m6),
            l8 = det * (m0 * m4 - m1 * m3);
    const R r0 = k * g.b0, r1 = k * g.b1, r2 = k * g.b2;
    ax = sc.invro * (l0 * r0 + l1 * r1 + l2 * r2);
    ay = sc.invro * (l3 * r0 + l4 * r1 + l5 * r2);
    az = sc.invro * (l6 * r0 + l7 * r1 + l8 * r2);
    return true;
}

// mirror part; the reference skips the mirror whose slot index equals i (kernel.cu:1759).
// Slots are stored as global_owner_id * NumMRR + k: the local slot is that minus
// NumMRR * pbase, the local particle index is pid_local.
template <class R, class RN, class G>
__device__ __forceinline__ void grad_sum_mirrors(const SceneDev<R, RN>& sc, const RowCtx<R>& c,
                                                 int pid_local, R x, R y, R z, R pmin,
                                                 const MirrorView<R>& m, bool skip, G& g,
                                                 int& cm) {
    const R B = skip ? sc.skip_rp : R(INFINITY);
    const int skip_slot = pid_local + kNumMRR * sc.pbase;
    for_rows(sc, m.cs, c, B, [&](int k) {
        if (__ldg(m.slot + k) == skip_slot) return;
        V4<R> q = ldg4(m.pos + k);
        R dx = q.x - x, dy = q.y - y, dz = q.z - z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 < sc.rp2) {
            R d = sqrtR(d2);
            g.add(wei_grad(d, sc.rp) / d2, q.w - pmin, dx, dy, dz);
            ++cm;
        }
    });
}

template <class R, class RN, class G>
__device__ __forceinline__ void grad_sum(const SceneDev<R, RN>& sc, const RowCtx<R>& c, int s,
                                         int pid_local, R x, R y, R z, R pi,
                                         const int* __restrict__ csr,
                                         const V4<R>* __restrict__ posf,
                                         const R* __restrict__ prs, const MirrorView<R>& m,
                                         bool skip, G& g, int& cf, int& cm) {
    R B = skip ? sc.skip_rp : R(INFINITY);
    R pmin = pi;
    for_fluid(sc, csr, posf, c, B, [&](int j, const V4<R>& q) {
        if (j == s) return;
        R dx = q.x - x, dy = q.y - y, dz = q.z - z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 < sc.rp2) {
            R pj = __ldg(prs + j);
            if (pj < pmin) pmin = pj;
        }
    });
    for_fluid(sc, csr, posf, c, B, [&](int j, const V4<R>& q) {
        if (j == s) return;
        R dx = q.x - x, dy = q.y - y, dz = q.z - z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 < sc.rp2) {
            R d = sqrtR(d2);
            g.add(wei_grad(d, sc.rp) / d2, __ldg(prs + j) - pmin, dx, dy, dz);
            ++cf;
        }
    });
    grad_sum_mirrors(sc, c, pid_local, x, y, z, pmin, m, skip, g, cm);
}

// ---- GenMRR_nonslip for one fluid particle (kernel.cu:726-891) ---------------------------
// In three parts, so that a warp reserves its mirrors' places in the raw list with one
// atomic: plan (registration over the walls inside r), count, emit.
template <class R> struct MirrorPlan {
    int nreg;    // registered normals: face mirror k comes from wall reg[k]
    int corner;  // wall whose position anchors the corner mirror, -1 when there is none
    int reg[kNumMRR];
    R sx, sy, sz;  // normalised sum of the distinct Edge normals
};

// A set of up to kNumMRR distinct normals in arrival order; the first three live in
// registers (walls meet a particle from one to three planes), the rest in a local array.
template <class R> struct NormalSet {
    int n = 0;
    R ax = R(0), ay = R(0), az = R(0), bx = R(0), by = R(0), bz = R(0), cx = R(0), cy = R(0),
      cz = R(0);
    R rest[kNumMRR - 3][3];
    __device__ __forceinline__ bool has(R x, R y, R z) const {
        if (n > 0 && ax == x && ay == y && az == z) return true;
        if (n > 1 && bx == x && by == y && bz == z) return true;
        if (n > 2 && cx == x && cy == y && cz == z) return true;
        for (int k = 3; k < n; ++k)
            if (rest[k - 3][0] == x && rest[k - 3][1] == y && rest[k - 3][2] == z) return true;
        return false;
    }
    __device__ __forceinline__ void add(R x, R y, R z) {
        if (n == 0) { ax = x; ay = y; az = z; }
        else if (n == 1) { bx = x; by = y; bz = z; }
        else if (n == 2) { cx = x; cy = y; cz = z; }
        else { rest[n - 3][0] = x; rest[n - 3][1] = y; rest[n - 3][2] = z; }
        ++n;
    }
    // component sums in arrival order
    __device__ __forceinline__ void sum(R& sx, R& sy, R& sz) const {
        sx = R(0); sy = R(0); sz = R(0);
        if (n > 0) { sx += ax; sy += ay; sz += az; }
        if (n > 1) { sx += bx; sy += by; sz += bz; }
        if (n > 2) { sx += cx; sy += cy; sz += cz; }
        for (int k = 3; k < n; ++k) { sx += rest[k - 3][0]; sy += rest[k - 3][1]; sz += rest[k - 3][2]; }
    }
};

// registration (kernel.cu:741-800): every distinct normal once, the first wall found wins;
// Edge walls likewise. Returns the number of walls inside r (diagnostic).
template <class R, class RN>
__device__ __forceinline__ int plan_mirrors(const SceneDev<R, RN>& sc, const RowCtx<R>& c, R x,
                                            R y, R z, const WallView<R>& wl, bool skip,
                                            MirrorPlan<R>& pl) {
    NormalSet<R> reg, edge;
    int last_edge = -1, nwall = 0;
    for_rows(sc, wl.cs, c, skip ? sc.skip_r : R(INFINITY), [&](int j) {
        V4<R> q = ldg4(wl.pos + j);
        R dx = x - q.x, dy = y - q.y, dz = z - q.z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (!(d2 <= sc.r2)) return;
        ++nwall;
        V4<R> nv = ldg4(wl.nrm + j);
        if (reg.n < kNumMRR && !reg.has(nv.x, nv.y, nv.z)) {
            pl.reg[reg.n] = j;
            reg.add(nv.x, nv.y, nv.z);
        }
        if (__ldg(wl.wse + j) == kEDGE && edge.n < kNumMRR && !edge.has(nv.x, nv.y, nv.z)) {
            last_edge = j;
            edge.add(nv.x, nv.y, nv.z);
        }
    });
    pl.nreg = reg.n;
    pl.corner = -1;
    // corner mirror through an Edge wall with the last registered Edge normal
    // (kernel.cu:841-858). The reference takes the first such wall its lists hold; with two
    // Edge normals (next to one edge of the tank) the nearest one is taken canonically, the
    // first found among equally near ones: it lies on that edge, the plane the reference's
    // runs pick there. Next to a vertex (three normals) the first one found stays.
    if (reg.n > 0 && edge.n >= 2) {
        R sx, sy, sz;
        edge.sum(sx, sy, sz);
        R as = sqrtR(dot3(sx, sy, sz, sx, sy, sz));
        pl.sx = sx / as; pl.sy = sy / as; pl.sz = sz / as;
        pl.corner = last_edge;
        if (edge.n == 2) {
            const V4<R> ln = ldg4(wl.nrm + last_edge);
            R best = R(INFINITY);
            for_rows(sc, wl.cs, c, skip ? sc.skip_r : R(INFINITY), [&](int j) {
                if (__ldg(wl.wse + j) != kEDGE) return;
                const V4<R> nv = ldg4(wl.nrm + j);
                if (nv.x != ln.x || nv.y != ln.y || nv.z != ln.z) return;
                const V4<R> q = ldg4(wl.pos + j);
                const R dx = x - q.x, dy = y - q.y, dz = z - q.z;
                const R d2 = dot3(dx, dy, dz, dx, dy, dz);
                if (d2 <= sc.r2 && d2 < best) {
                    best = d2;
                    pl.corner = j;
                }
            });
        }
    }
    return nwall;
}

// mirrors the plan will emit; a corner mirror without a free slot is counted as an error
// (kernel.cu:868-874 writes it out of bounds)
template <class R, class RN>
__device__ __forceinline__ int count_mirrors(const MirrorPlan<R>& pl, R x, R y, R z,
                                             const WallView<R>& wl, DevCounters* cnt) {
    int m = 0;
    for (int k = 0; k < pl.nreg; ++k) {
        V4<R> q = ldg4(wl.pos + pl.reg[k]), n = ldg4(wl.nrm + pl.reg[k]);
        if (!(dot3(x - q.x, y - q.y, z - q.z, n.x, n.y, n.z) < R(0))) ++m;
    }
    if (pl.corner >= 0) {
        V4<R> q = ldg4(wl.pos + pl.corner);
        if (dot3(x - q.x, y - q.y, z - q.z, pl.sx, pl.sy, pl.sz) >= R(0)) {
            if (pl.nreg >= kNumMRR) atomicAdd(&cnt->err_mirror_slot, 1);
            else ++m;
        }
    }
    return m;
}

// face mirrors (kernel.cu:811-838), then the corner mirror (kernel.cu:859-887), written to
// the raw list from index `at` on
template <class R, class RN, bool TAPE>
__device__ __forceinline__ void emit_mirrors(const MirrorPlan<R>& pl, R x, R y, R z, R P,
                                             int slot_base, const WallView<R>& wl,
                                             const MirrorSink<R>& out, DevCounters* cnt, int at) {
    auto emit = [&](R mx, R my, R mz, int slot, R nx, R ny, R nz, R nlen) {
        const int idx = at++;
        if (idx < out.cap) {
            out.pos[idx] = V4<R>{mx, my, mz, P};
            out.slot[idx] = slot;
            if (TAPE) {
                const R cf = sqrtR(R(2) / nlen);
                out.nrm[idx] = V4<R>{nx * cf, ny * cf, nz * cf, R(0)};
            }
        } else {
            atomicAdd(&cnt->err_capacity, 1);
        }
    };
    for (int k = 0; k < pl.nreg; ++k) {
        V4<R> q = ldg4(wl.pos + pl.reg[k]), n = ldg4(wl.nrm + pl.reg[k]);
        R pwx = x - q.x, pwy = y - q.y, pwz = z - q.z;
        R pw = dot3(pwx, pwy, pwz, n.x, n.y, n.z);
        if (pw < R(0)) continue;
        R nlen = sqrtR(dot3(n.x, n.y, n.z, n.x, n.y, n.z));
        R dist = pw / nlen;
        R t2 = R(2) * dist;
        emit(fmaR(-t2, n.x, q.x + pwx), fmaR(-t2, n.y, q.y + pwy), fmaR(-t2, n.z, q.z + pwz),
             slot_base + k, n.x, n.y, n.z, nlen);
    }
    if (pl.corner >= 0 && pl.nreg < kNumMRR) {
        V4<R> q = ldg4(wl.pos + pl.corner);
        R pwx = x - q.x, pwy = y - q.y, pwz = z - q.z;
        R pw = dot3(pwx, pwy, pwz, pl.sx, pl.sy, pl.sz);
        if (pw >= R(0)) {
            R slen = sqrtR(dot3(pl.sx, pl.sy, pl.sz, pl.sx, pl.sy, pl.sz));
            R dist = pw / slen;
            R t2 = R(2) * dist;
            emit(fmaR(-t2, pl.sx, q.x + pwx), fmaR(-t2, pl.sy, q.y + pwy),
                 fmaR(-t2, pl.sz, q.z + pwz), slot_base + pl.nreg, pl.sx, pl.sy, pl.sz, slen);
        }
    }
}

}  // namespace mps
