// mps_oracle.cpp -- CPU oracle of the explicit MPS step (TEST INFRASTRUCTURE ONLY).
//
// Restates the per-particle loop bodies of frsykzk/MPS_CUDA kernel.cu for the checks in
// tests/, the cpu_baseline leg of bench.py and bench.py's reference arm. The product
// (mps_cuda_b200) never links or calls this file.
//
// What is restated, and from where (file:line in the reference project):
//   constants, weights          const.cuh:27-53
//   AlcBkt / SetPara            kernel.cu:307-373   (+ explicit snd/dt/umax/pmax)
//   bucket index                kernel.cu:521-524
//   Surface_Edge                kernel.cu:553-668
//   ResetMRR / GenMRR_nonslip   kernel.cu:691-893
//   MkBkt_MRR / MRRinout        kernel.cu:916-1010
//   VscTrm                      kernel.cu:1013-1119
//   UpPcl1 + ChkPcl             kernel.cu:1138-1149, 481-513
//   ChkCol + UpChkCol           kernel.cu:1168-1287
//   MkPrs                       kernel.cu:1306-1411
//   PrsGrdTrm (active variant)  kernel.cu:1651-1794
//   UpPcl2                      kernel.cu:1815-1829
//   step order                  kernel.cu:1904-1941
//
// Canonical choices that the reference leaves open (its atomicExch linked lists give a
// run-to-run varying neighbour order, kernel.cu:525-527):
//   * bucket lists are ordered by ascending particle id (mirror slot id for mirrors);
//     the 27 buckets are walked z, y, x ascending as in every reference loop;
//   * fluid neighbours are visited in fine cells, a third of a bucket per axis and nested
//     in the buckets (fine x = int(3 t) + 3 with t the bucket coordinate): the 9 x 9 x 9
//     fine cells of the 27 buckets z, y, x ascending, ascending id inside a fine cell.
//     The candidates are the reference's (the particles of the 27 buckets); only the
//     order of the sums is fixed this way;
//   * ChkCol visits fluid neighbours, then wall neighbours, then mirrors;
//   * with two distinct Edge normals in reach, the corner mirror's plane point is the
//     NEAREST Edge wall with the last registered Edge normal, where the reference takes the
//     first one its lists hold (kernel.cu:852-858): near a tank edge that is a wall on the
//     edge itself, the plane the reference's runs choose there, while the first wall in id
//     order can lie on another border of the face;
//   * arithmetic is written with explicit fma where a product feeds a sum (the forms an
//     FMA-contracting compiler produces) and is built with -ffp-contract=off, so every
//     expression rounds the same way on every machine;
//   * VscTrm uses w = 2 l0 / (dist2 * dist) for 2 l0 / dist / dist / dist;
//   * the corner mirror's synvec starts at zero (kernel.cu:849 leaves it uninitialised);
//   * a corner mirror without a free slot is counted, not written (kernel.cu:868-874).
#include "mps_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int GST = -1, FLD = 0, WLL = 1, OBJ = 2, OBJ2 = 3, MRR = 4;
constexpr int EDGE = 1;
constexpr int NUM_MRR = 10;
enum {
    PH_MKBKT = 0, PH_SURFACE_EDGE, PH_RESETMRR, PH_GENMRR, PH_MKBKT_MRR, PH_VSCTRM,
    PH_UPPCL1, PH_CHKCOL, PH_MKPRS, PH_PRSGRDTRM, PH_UPPCL2
};
enum { D_CELL = 0, D_VSC_F, D_VSC_M, D_COL_F, D_COL_W, D_COL_M, D_PRS_F, D_PRS_M, D_GRD_F,
       D_GRD_M, D_GEN_W, D_NCOL };

inline bool is_wall(int t) { return t == WLL || t == OBJ || t == OBJ2; }

template <class R> inline R fmar(R a, R b, R c) { return std::fma(a, b, c); }
// |p|^2 in the canonical form fma(z, z, fma(y, y, x*x)).
template <class R> inline R dot3(R ax, R ay, R az, R bx, R by, R bz) {
    return fmar(az, bz, fmar(ay, by, ax * bx));
}
// WEI / WEI_grad, const.cuh:45-46
template <class R> inline R wei(R d, R re) { return ((re / d) + (d / re)) - R(2); }
template <class R> inline R wei_grad(R d, R re) { return (re / d) - (d / re); }

template <class R, class RN>
struct Oracle {
    // ---- parameters, AlcBkt / SetPara (kernel.cu:307-373) -----------------------------
    R l0, r, r2, rp, rp2, db, dbinv;
    R minc[3], maxc[3], lo[3], hi[3], g[3];
    int nbx, nby, nbz, nbxy, nbxyz;
    int nfx, nfy, nfz, nfxy, nfxyz;  // fine cells: a third of a bucket per axis
    R n0, lmd, n0_grad, lmd_grad;
    int numn0_grad;
    RN n0_grad_n, prs_coef_n, pmax_n, rho_n;
    R rlim2, col, rho, knm, snd, prs_coef, pmax, umax, dt, rlim_wall2, edge_r2;
    int grad_mode = 0;  // 0: PrsGrdTrm as compiled (kernel.cu:1651-1794), 1: the #if 0 variant
    // prescribed motion of OBJ (0) and OBJ2 (1) walls: a wall set moving at x0 with normal n0
    // is at c + t + q (x0 - c), normal q n0, velocity v + w x (q (x0 - c)); q and t gather
    // one step's rotation qs (omega dt about the unit axis, Rodrigues) and translation v dt
    struct Motion {
        int type = 0;
        double qs[9], q[9], c[3], t[3], vdt[3], w[3], v[3];
    } mot[2];
    std::vector<double> mx0, mn0;  // reference state of moving walls, SoA by particle id

    int n;
    std::vector<int8_t> typ, wse;
    std::vector<R> px, py, pz, vx, vy, vz, ax, ay, az, prs, pav, nx, ny, nz;
    // mirror slots, reference layout d_TypM / d_PosM / d_VelM / d_PrsM (kernel.cu:96-103)
    std::vector<int8_t> mtyp;
    std::vector<R> mx, my, mz, mvx, mvy, mvz, mprs;
    // bucket lists: particles (fluid + walls, not GST) and mirrors, ascending id per bucket
    std::vector<int> cstart, clist, mstart, mlist, cell_of;
    // fluid lists over fine cells, ascending id per fine cell
    std::vector<int> fstart, flist;
    // diagnostics
    std::vector<int32_t> diag;
    std::vector<R> ndens;

    void derive(const oracle_params& p) {
        l0 = R(p.pcl_dst);
        // RdDat pads the domain by 3.1 l0 in double and rounds to real (kernel.cu:25-31)
        for (int d = 0; d < 3; ++d) {
            R mn = R(p.min[d]), mx_ = R(p.max[d]);
            minc[d] = R(double(mn) - 3.1 * double(l0));
            maxc[d] = R(double(mx_) + 3.1 * double(l0));
            g[d] = R(p.g[d]);
        }
        // AlcBkt, kernel.cu:309-322
        r = l0 * R(3.1);
        r2 = r * r;
        rp = l0 * R(2.1);
        rp2 = rp * rp;
        db = l0 * R(3.1);
        dbinv = R(1) / db;
        nbx = int((maxc[0] - minc[0]) * dbinv) + 3;
        nby = int((maxc[1] - minc[1]) * dbinv) + 3;
        nbz = int((maxc[2] - minc[2]) * dbinv) + 3;
        nbxy = nbx * nby;
        nbxyz = nbxy * nbz;
        nfx = 3 * nbx;
        nfy = 3 * nby;
        nfz = 3 * nbz;
        nfxy = nfx * nfy;
        nfxyz = nfxy * nfz;
        // SetPara lattice sums, kernel.cu:336-366
        R tn0 = 0, tn0g = 0, tl = 0, tlg = 0;
        int cnt = 0;
        for (int ix = -10; ix < 10; ++ix)
            for (int iy = -10; iy < 10; ++iy)
                for (int iz = -10; iz < 10; ++iz) {
                    R x = l0 * R(ix), y = l0 * R(iy), z = l0 * R(iz);
                    R d2 = x * x + y * y + z * z;
                    if (d2 == R(0)) continue;
                    R d = std::sqrt(d2);
                    if (d2 < rp2) {
                        tn0g += wei_grad(d, rp);
                        tlg += d2 * wei_grad(d, rp);
                        cnt += 1;
                    }
                    if (d2 < r2) {
                        tn0 += wei(d, r);
                        tl += d2 * wei(d, r);
                    }
                }
        n0 = tn0;
        lmd = tl / tn0;
        n0_grad = tn0g;
        lmd_grad = tlg / tn0g;
        numn0_grad = cnt;
        // kernel.cu:370-373
        R rlim = l0 * R(p.dst_lmt_rat);
        rlim2 = rlim * rlim;
        col = R(p.col_rat) + R(1);
        rho = R(p.rho);
        knm = R(p.knm_vsc);
        snd = R(p.snd);
        prs_coef = snd * snd / n0_grad;  // kernel.cu:409
        pmax = R(p.pmax);
        umax = R(p.umax);
        dt = R(p.dt);
        R rlim_wall = R(0.45) * l0;  // kernel.cu:1184-1185
        rlim_wall2 = rlim_wall * rlim_wall;
        edge_r2 = (R(1) * l0) * (R(1) * l0);  // kernel.cu:558
        // ChkPcl box, kernel.cu:484-486
        for (int d = 0; d < 3; ++d) {
            R t = R(3.1) * l0;
            lo[d] = minc[d] + t;
            hi[d] = maxc[d] - t;
        }
        // number-density arithmetic (double in the mixed mode)
        if (sizeof(RN) == sizeof(R)) {
            n0_grad_n = RN(n0_grad);
        } else {
            RN s = 0, l0n = RN(l0), rpn = RN(rp), rp2n = rpn * rpn;
            for (int ix = -10; ix < 10; ++ix)
                for (int iy = -10; iy < 10; ++iy)
                    for (int iz = -10; iz < 10; ++iz) {
                        RN x = l0n * RN(ix), y = l0n * RN(iy), z = l0n * RN(iz);
                        RN d2 = x * x + y * y + z * z;
                        if (d2 == RN(0)) continue;
                        if (d2 < rp2n) s += wei_grad(std::sqrt(d2), rpn);
                    }
            n0_grad_n = s;
        }
        prs_coef_n = RN(snd) * RN(snd) / n0_grad_n;
        pmax_n = RN(pmax);
        rho_n = RN(rho);
    }

    // bucket index, kernel.cu:521-524
    inline int cell3(R x, R y, R z, int& ix, int& iy, int& iz) const {
        ix = int((x - minc[0]) * dbinv) + 1;
        iy = int((y - minc[1]) * dbinv) + 1;
        iz = int((z - minc[2]) * dbinv) + 1;
        return iz * nbxy + iy * nbx + ix;
    }
    // fine cell inside bucket (ix, iy, iz): fx = int(3 t) + 3, t = (x - minc) * dbinv
    inline int fine3(R x, R y, R z, int ix, int iy, int iz) const {
        const R tx = (x - minc[0]) * dbinv, ty = (y - minc[1]) * dbinv, tz = (z - minc[2]) * dbinv;
        const int fx = std::min(std::max(int(R(3) * tx) + 3, 3 * ix), 3 * ix + 2);
        const int fy = std::min(std::max(int(R(3) * ty) + 3, 3 * iy), 3 * iy + 2);
        const int fz = std::min(std::max(int(R(3) * tz) + 3, 3 * iz), 3 * iz + 2);
        return fz * nfxy + fy * nfx + fx;
    }
    inline bool cell_ok(int ix, int iy, int iz) const {
        return ix >= 1 && ix <= nbx - 2 && iy >= 1 && iy <= nby - 2 && iz >= 1 && iz <= nbz - 2;
    }

    void init(const oracle_params& p, int n_, const int8_t* t, const R* pos, const R* vel,
              const R* nrm) {
        derive(p);
        n = n_;
        typ.assign(t, t + n);
        px.assign(pos, pos + n); py.assign(pos + n, pos + 2 * n); pz.assign(pos + 2 * n, pos + 3 * n);
        vx.assign(vel, vel + n); vy.assign(vel + n, vel + 2 * n); vz.assign(vel + 2 * n, vel + 3 * n);
        nx.assign(nrm, nrm + n); ny.assign(nrm + n, nrm + 2 * n); nz.assign(nrm + 2 * n, nrm + 3 * n);
        ax.assign(n, R(0)); ay.assign(n, R(0)); az.assign(n, R(0));
        prs.assign(n, R(0)); pav.assign(n, R(0));
        wse.assign(n, 0);
        // RdDat keeps only particles inside the padded box (kernel.cu:117)
        for (int i = 0; i < n; ++i) {
            bool in = px[i] < maxc[0] && px[i] > minc[0] && py[i] < maxc[1] && py[i] > minc[1] &&
                      pz[i] < maxc[2] && pz[i] > minc[2];
            if (!in) typ[i] = GST;
            if (typ[i] == FLD || typ[i] == GST) { nx[i] = ny[i] = nz[i] = R(0); }
        }
        size_t nm = size_t(n) * NUM_MRR;
        mtyp.assign(nm, int8_t(GST));
        mx.assign(nm, R(0)); my.assign(nm, R(0)); mz.assign(nm, R(0));
        mvx.assign(nm, R(0)); mvy.assign(nm, R(0)); mvz.assign(nm, R(0)); mprs.assign(nm, R(0));
        diag.assign(size_t(n) * D_NCOL, 0);
        ndens.assign(n, R(0));
        cell_of.assign(n, -1);
        mstart.assign(nbxyz + 1, 0);
        // ClcMPS starts with MkBkt + Surface_Edge (kernel.cu:1878-1879)
        mkbkt();
        surface_edge();
    }

    // ---- MkBkt (kernel.cu:516-550): ordered bucket lists ------------------------------
    void mkbkt() {
        cstart.assign(nbxyz + 1, 0);
        for (int i = 0; i < n; ++i) {
            int c = -1;
            if (typ[i] != GST) {
                int ix, iy, iz;
                c = cell3(px[i], py[i], pz[i], ix, iy, iz);
                if (c < 0 || c >= nbxyz) c = -1;
            }
            cell_of[i] = c;
            if (c >= 0) cstart[c + 1]++;
        }
        for (int c = 0; c < nbxyz; ++c) cstart[c + 1] += cstart[c];
        clist.assign(cstart[nbxyz], 0);
        std::vector<int> fill(cstart.begin(), cstart.end() - 1);
        for (int i = 0; i < n; ++i)
            if (cell_of[i] >= 0) clist[fill[cell_of[i]]++] = i;
        // fluid by fine cell
        fstart.assign(size_t(nfxyz) + 1, 0);
        std::vector<int> fc(n, -1);
        for (int i = 0; i < n; ++i) {
            if (typ[i] != FLD || cell_of[i] < 0) continue;
            int ix, iy, iz;
            cell3(px[i], py[i], pz[i], ix, iy, iz);
            fc[i] = fine3(px[i], py[i], pz[i], ix, iy, iz);
            fstart[fc[i] + 1]++;
        }
        for (int c = 0; c < nfxyz; ++c) fstart[c + 1] += fstart[c];
        flist.assign(fstart[nfxyz], 0);
        std::vector<int> ffill(fstart.begin(), fstart.end() - 1);
        for (int i = 0; i < n; ++i)
            if (fc[i] >= 0) flist[ffill[fc[i]]++] = i;
    }

    // mirror list over MRR slots in ascending slot order (d_MkBkt_MRR, kernel.cu:916-929)
    void mkbkt_mrr() {
        mstart.assign(nbxyz + 1, 0);
        size_t nm = mtyp.size();
        std::vector<int> mc(nm, -1);
        for (size_t s = 0; s < nm; ++s) {
            if (mtyp[s] == GST) continue;
            int ix, iy, iz;
            int c = cell3(mx[s], my[s], mz[s], ix, iy, iz);
            if (c < 0 || c >= nbxyz) continue;
            mc[s] = c;
            mstart[c + 1]++;
        }
        for (int c = 0; c < nbxyz; ++c) mstart[c + 1] += mstart[c];
        mlist.assign(mstart[nbxyz], 0);
        std::vector<int> fill(mstart.begin(), mstart.end() - 1);
        for (size_t s = 0; s < nm; ++s)
            if (mc[s] >= 0) mlist[fill[mc[s]]++] = int(s);
    }

    // visit the 27 buckets around (ix, iy, iz), z then y then x ascending
    template <class F> inline void for_nb(const std::vector<int>& st, const std::vector<int>& li,
                                          int ix, int iy, int iz, F&& f) const {
        for (int jz = iz - 1; jz <= iz + 1; ++jz)
            for (int jy = iy - 1; jy <= iy + 1; ++jy)
                for (int jx = ix - 1; jx <= ix + 1; ++jx) {
                    if (jx < 0 || jy < 0 || jz < 0 || jx >= nbx || jy >= nby || jz >= nbz) continue;
                    int jb = jz * nbxy + jy * nbx + jx;
                    for (int k = st[jb]; k < st[jb + 1]; ++k) f(li[k]);
                }
    }

    // visit the fluid of the 27 buckets around (ix, iy, iz) in fine cells, z, y, x
    // ascending; fine cells farther than radius (+ 1e-3 of a bucket) from (x, y, z) hold no
    // neighbour and are passed over
    template <class F> inline void for_fluid(R x, R y, R z, int ix, int iy, int iz, R radius,
                                             F&& f) const {
        const double h = 1.0 / (3.0 * double(dbinv)), m = double(radius) + 1e-3 * double(db);
        const double rx = double(x) - double(minc[0]), ry = double(y) - double(minc[1]),
                     rz = double(z) - double(minc[2]);
        auto gap = [&](double v, int fc) {
            const double a = (fc - 3) * h;
            return std::max({a - v, v - (a + h), 0.0});
        };
        for (int fz = 3 * iz - 3; fz <= 3 * iz + 5; ++fz) {
            if (fz < 0 || fz >= nfz) continue;
            const double gz = gap(rz, fz);
            for (int fy = 3 * iy - 3; fy <= 3 * iy + 5; ++fy) {
                if (fy < 0 || fy >= nfy) continue;
                const double gy = gap(ry, fy);
                if (gy * gy + gz * gz > m * m) continue;
                for (int fx = 3 * ix - 3; fx <= 3 * ix + 5; ++fx) {
                    if (fx < 0 || fx >= nfx) continue;
                    const double gx = gap(rx, fx);
                    if (gx * gx + gy * gy + gz * gz > m * m) continue;
                    const int c = fz * nfxy + fy * nfx + fx;
                    for (int k = fstart[c]; k < fstart[c + 1]; ++k) f(flist[k]);
                }
            }
        }
    }

    // ---- Surface_Edge (kernel.cu:553-668) ----------------------------------------------
    void surface_edge() {
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            int t = typ[i];
            if (!is_wall(t)) continue;
            int ix, iy, iz;
            cell3(px[i], py[i], pz[i], ix, iy, iz);
            bool edge = false;
            for_nb(cstart, clist, ix, iy, iz, [&](int j) {
                if (j == i || typ[j] != t) return;
                R d2 = dot3(px[i] - px[j], py[i] - py[j], pz[i] - pz[j], px[i] - px[j],
                            py[i] - py[j], pz[i] - pz[j]);
                if (d2 < edge_r2) {
                    if (nx[j] != nx[i] || ny[j] != ny[i] || nz[j] != nz[i]) edge = true;
                }
            });
            if (edge) wse[i] = EDGE;
        }
    }

    // ---- ResetMRR (kernel.cu:691-701) ---------------------------------------------------
    void reset_mrr() {
        std::fill(mtyp.begin(), mtyp.end(), int8_t(GST));
        std::fill(mx.begin(), mx.end(), R(0)); std::fill(my.begin(), my.end(), R(0));
        std::fill(mz.begin(), mz.end(), R(0)); std::fill(mvx.begin(), mvx.end(), R(0));
        std::fill(mvy.begin(), mvy.end(), R(0)); std::fill(mvz.begin(), mvz.end(), R(0));
        std::fill(mprs.begin(), mprs.end(), R(0));
    }

    int err_mirror_slot = 0;

    // ---- GenMRR_nonslip (kernel.cu:720-893) ----------------------------------------------
    void gen_mrr() {
        int errs = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : errs)
        for (int i = 0; i < n; ++i) {
            if (typ[i] != FLD) continue;
            R x = px[i], y = py[i], z = pz[i];
            int from[NUM_MRR], edgeu[NUM_MRR];
            int nreg = 0, nedge = 0, ngen = 0;
            int ix, iy, iz;
            cell3(x, y, z, ix, iy, iz);
            for_nb(cstart, clist, ix, iy, iz, [&](int j) {
                if (j == i || !is_wall(typ[j])) return;
                R qx = x - px[j], qy = y - py[j], qz = z - pz[j];
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (!(d2 <= r2)) return;
                ++ngen;
                // register each distinct normal once; the first wall found wins (:758-775)
                bool dup = false;
                for (int k = 0; k < nreg; ++k) {
                    int q = from[k];
                    if (nx[q] == nx[j] && ny[q] == ny[j] && nz[q] == nz[j]) dup = true;
                }
                if (!dup && nreg < NUM_MRR) from[nreg++] = j;
                if (wse[j] == EDGE) {  // (:777-796)
                    bool edup = false;
                    for (int k = 0; k < nedge; ++k) {
                        int q = edgeu[k];
                        if (nx[q] == nx[j] && ny[q] == ny[j] && nz[q] == nz[j]) edup = true;
                    }
                    if (!edup && nedge < NUM_MRR) edgeu[nedge++] = j;
                }
            });
            diag[size_t(i) * D_NCOL + D_GEN_W] = ngen;
            if (nreg == 0) continue;
            size_t base = size_t(i) * NUM_MRR;
            // face mirrors (:811-838)
            for (int k = 0; k < nreg; ++k) {
                int w = from[k];
                R pwx = x - px[w], pwy = y - py[w], pwz = z - pz[w];
                R pw = dot3(pwx, pwy, pwz, nx[w], ny[w], nz[w]);
                if (pw < R(0)) continue;
                R dist = pw / std::sqrt(dot3(nx[w], ny[w], nz[w], nx[w], ny[w], nz[w]));
                R t2 = R(2) * dist;
                size_t s = base + k;
                mtyp[s] = MRR;
                mx[s] = fmar(-t2, nx[w], px[w] + pwx);
                my[s] = fmar(-t2, ny[w], py[w] + pwy);
                mz[s] = fmar(-t2, nz[w], pz[w] + pwz);
                mprs[s] = prs[i];
                mvx[s] = mvy[s] = mvz[s] = R(0);
            }
            // corner mirror from the normalised sum of edge normals (:841-887)
            if (nedge >= 2) {
                // Its plane point: an Edge wall with the last registered Edge normal. The
                // reference takes the first such wall its linked lists happen to hold
                // (:852-858), an order that changes with thread scheduling. With two Edge
                // normals (a particle next to one edge of the tank) the nearest such wall is
                // taken canonically (the first found among equally near ones): it lies on
                // that edge, the plane the reference's runs pick there. Next to a vertex
                // (three normals) the first one in visiting order stays.
                const int wl = edgeu[nedge - 1];
                int best = wl;
                R best_d2 = R(INFINITY);
                if (nedge == 2) for_nb(cstart, clist, ix, iy, iz, [&](int j) {
                    if (!is_wall(typ[j]) || wse[j] != EDGE) return;
                    if (nx[j] != nx[wl] || ny[j] != ny[wl] || nz[j] != nz[wl]) return;
                    R qx = x - px[j], qy = y - py[j], qz = z - pz[j];
                    R d2 = dot3(qx, qy, qz, qx, qy, qz);
                    if (d2 <= r2 && d2 < best_d2) { best_d2 = d2; best = j; }
                });
                edgeu[nedge - 1] = best;
                R sx = 0, sy = 0, sz = 0, pwx = 0, pwy = 0, pwz = 0, wx = 0, wy = 0, wz = 0;
                for (int k = 0; k < nedge; ++k) {
                    int w = edgeu[k];
                    wx = px[w]; wy = py[w]; wz = pz[w];
                    sx += nx[w]; sy += ny[w]; sz += nz[w];
                    pwx = x - wx; pwy = y - wy; pwz = z - wz;
                }
                R as = std::sqrt(dot3(sx, sy, sz, sx, sy, sz));
                sx /= as; sy /= as; sz /= as;
                R pw = dot3(pwx, pwy, pwz, sx, sy, sz);
                if (pw < R(0)) continue;
                R dist = pw / std::sqrt(dot3(sx, sy, sz, sx, sy, sz));
                if (nreg >= NUM_MRR) { ++errs; continue; }
                R t2 = R(2) * dist;
                size_t s = base + nreg;
                mtyp[s] = MRR;
                mx[s] = fmar(-t2, sx, wx + pwx);
                my[s] = fmar(-t2, sy, wy + pwy);
                mz[s] = fmar(-t2, sz, wz + pwz);
                mvx[s] = mvy[s] = mvz[s] = R(0);
                mprs[s] = prs[i];
            }
        }
        err_mirror_slot += errs;
    }

    // ---- MkBkt_MRR: MRRinout cull + mirror list (kernel.cu:932-1010) ----------------------
    void mkbkt_mrr_phase() {
        size_t nm = mtyp.size();
#pragma omp parallel for schedule(dynamic, 1024)
        for (long long s = 0; s < (long long)nm; ++s) {
            if (mtyp[s] == GST) continue;  // the reference also visits GST slots: no effect
            R x = mx[s], y = my[s], z = mz[s];
            int ix, iy, iz;
            cell3(x, y, z, ix, iy, iz);
            bool found = false;
            R walldist = R(10) * r;
            R wx = 0, wy = 0, wz = 0, vx_ = 0, vy_ = 0, vz_ = 0;
            for_nb(cstart, clist, ix, iy, iz, [&](int j) {
                if (!is_wall(typ[j])) return;
                R qx = x - px[j], qy = y - py[j], qz = z - pz[j];
                R d = std::sqrt(dot3(qx, qy, qz, qx, qy, qz));
                if (d <= r) {
                    if (d < walldist) {
                        found = true;
                        walldist = d;
                        vx_ = nx[j]; vy_ = ny[j]; vz_ = nz[j];
                        wx = px[j]; wy = py[j]; wz = pz[j];
                    }
                }
            });
            R inout = dot3(x - wx, y - wy, z - wz, vx_, vy_, vz_);
            if (found && inout >= R(0)) mtyp[s] = GST;
        }
        mkbkt_mrr();
    }

    // ---- VscTrm (kernel.cu:1013-1119) --------------------------------------------------
    void vsctrm() {
        const R two_l0 = R(2) * l0;
        const R kn = (R(1) / n0) * knm;
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (typ[i] != FLD) continue;
            R x = px[i], y = py[i], z = pz[i], ux = vx[i], uy = vy[i], uz = vz[i];
            R sx = 0, sy = 0, sz = 0;
            int cf = 0, cm = 0;
            int ix, iy, iz;
            cell3(x, y, z, ix, iy, iz);
            for_fluid(x, y, z, ix, iy, iz, r, [&](int j) {
                if (j == i || typ[j] != FLD) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                R d = std::sqrt(d2);
                if (d <= r) {
                    R w = two_l0 / (d2 * d);
                    sx = fmar(vx[j] - ux, w, sx);
                    sy = fmar(vy[j] - uy, w, sy);
                    sz = fmar(vz[j] - uz, w, sz);
                    ++cf;
                }
            });
            for_nb(mstart, mlist, ix, iy, iz, [&](int s) {
                R qx = mx[s] - x, qy = my[s] - y, qz = mz[s] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                R d = std::sqrt(d2);
                if (d <= r) {
                    R w = two_l0 / (d2 * d);
                    sx = fmar(mvx[s] - ux, w, sx);
                    sy = fmar(mvy[s] - uy, w, sy);
                    sz = fmar(mvz[s] - uz, w, sz);
                    ++cm;
                }
            });
            ax[i] = fmar(kn, sx, g[0]);
            ay[i] = fmar(kn, sy, g[1]);
            az[i] = fmar(kn, sz, g[2]);
            diag[size_t(i) * D_NCOL + D_VSC_F] = cf;
            diag[size_t(i) * D_NCOL + D_VSC_M] = cm;
        }
    }

    // ---- ChkPcl (kernel.cu:481-513) ----------------------------------------------------
    inline void chkpcl(int i) {
        if (typ[i] != FLD) return;
        if (px[i] < hi[0] && px[i] > lo[0] && py[i] < hi[1] && py[i] > lo[1] && pz[i] < hi[2] &&
            pz[i] > lo[2]) {
            R u = std::sqrt(dot3(vx[i], vy[i], vz[i], vx[i], vy[i], vz[i]));
            if (u > umax) {
                R s = umax / u;
                vx[i] *= s; vy[i] *= s; vz[i] *= s;
            }
        } else {
            typ[i] = GST;
            px[i] = py[i] = pz[i] = R(0);
            vx[i] = vy[i] = vz[i] = R(0);
            ax[i] = ay[i] = az[i] = R(0);
            prs[i] = R(0);
        }
    }

    // ---- UpPcl1 (kernel.cu:1138-1149) ----------------------------------------------------
    void uppcl1() {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            if (typ[i] == FLD) {
                vx[i] = fmar(ax[i], dt, vx[i]); vy[i] = fmar(ay[i], dt, vy[i]); vz[i] = fmar(az[i], dt, vz[i]);
                px[i] = fmar(vx[i], dt, px[i]); py[i] = fmar(vy[i], dt, py[i]); pz[i] = fmar(vz[i], dt, pz[i]);
                ax[i] = ay[i] = az[i] = R(0);
            }
            chkpcl(i);
        }
    }

    // ---- ChkCol + UpChkCol (kernel.cu:1168-1287) ------------------------------------------
    void chkcol() {
        const R colfac = (col * rho) / (rho + rho);
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (typ[i] != FLD) continue;
            R x = px[i], y = py[i], z = pz[i];
            R ux = vx[i], uy = vy[i], uz = vz[i];
            R wx = ux, wy = uy, wz = uz;
            int cf = 0, cw = 0, cm = 0;
            int ix, iy, iz;
            cell3(x, y, z, ix, iy, iz);
            auto hit = [&](R qx, R qy, R qz, R d2, R jx, R jy, R jz) {
                R f = dot3(ux - jx, uy - jy, uz - jz, qx, qy, qz);
                if (f > R(0)) {
                    f = f * (colfac / d2);
                    wx = fmar(-qx, f, wx); wy = fmar(-qy, f, wy); wz = fmar(-qz, f, wz);
                }
            };
            for_fluid(x, y, z, ix, iy, iz, std::sqrt(rlim2), [&](int j) {
                if (j == i || typ[j] != FLD) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rlim2) { ++cf; hit(qx, qy, qz, d2, vx[j], vy[j], vz[j]); }
            });
            for_nb(cstart, clist, ix, iy, iz, [&](int j) {
                if (!is_wall(typ[j])) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rlim_wall2) { ++cw; hit(qx, qy, qz, d2, vx[j], vy[j], vz[j]); }
            });
            for_nb(mstart, mlist, ix, iy, iz, [&](int s) {
                R qx = mx[s] - x, qy = my[s] - y, qz = mz[s] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rlim2) { ++cm; hit(qx, qy, qz, d2, mvx[s], mvy[s], mvz[s]); }
            });
            ax[i] = wx; ay[i] = wy; az[i] = wz;
            diag[size_t(i) * D_NCOL + D_COL_F] = cf;
            diag[size_t(i) * D_NCOL + D_COL_W] = cw;
            diag[size_t(i) * D_NCOL + D_COL_M] = cm;
        }
        // d_UpChkCol (kernel.cu:1281-1287)
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i)
            if (typ[i] == FLD) { vx[i] = ax[i]; vy[i] = ay[i]; vz[i] = az[i]; }
    }

    // ---- MkPrs (kernel.cu:1306-1411) -----------------------------------------------------
    void mkprs() {
        const RN rpn = RN(rp);
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (typ[i] != FLD) continue;
            R x = px[i], y = py[i], z = pz[i];
            RN ni = 0;
            int cf = 0, cm = 0;
            int ix, iy, iz;
            cell3(x, y, z, ix, iy, iz);
            auto add = [&](R d2) {
                R d = std::sqrt(d2);
                if (d < rp) {
                    RN dn = (sizeof(RN) == sizeof(R)) ? RN(d) : std::sqrt(RN(d2));
                    ni += wei_grad(dn, rpn);
                    return true;
                }
                return false;
            };
            for_fluid(x, y, z, ix, iy, iz, rp, [&](int j) {
                if (j == i || typ[j] != FLD) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                if (add(dot3(qx, qy, qz, qx, qy, qz))) ++cf;
            });
            for_nb(mstart, mlist, ix, iy, iz, [&](int s) {
                R qx = mx[s] - x, qy = my[s] - y, qz = mz[s] - z;
                if (add(dot3(qx, qy, qz, qx, qy, qz))) ++cm;
            });
            RN pr = RN(ni > n0_grad_n ? 1 : 0) * (ni - n0_grad_n) * prs_coef_n * rho_n;
            if (pr <= pmax_n && pr >= RN(0)) {
            } else {
                pr = (pr > pmax_n) ? pmax_n : RN(0);
            }
            prs[i] = R(pr);
            ndens[i] = R(ni);
            diag[size_t(i) * D_NCOL + D_PRS_F] = cf;
            diag[size_t(i) * D_NCOL + D_PRS_M] = cm;
        }
    }

    // ---- moving walls ---------------------------------------------------------------------
    int set_motion(int type, const double* c, const double* axis, double omega, const double* v) {
        if (type != OBJ && type != OBJ2) return 1;
        Motion w;
        double a[3] = {0.0, 0.0, 1.0};
        if (omega != 0.0) {
            const double nn = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
            if (!(nn > 0.0)) return 1;
            for (int d = 0; d < 3; ++d) a[d] = axis[d] / nn;
        }
        const double step = double(dt);
        const double th = omega * step, cs = std::cos(th), sn = std::sin(th), cc = 1.0 - cs;
        const double qs[9] = {cs + a[0] * a[0] * cc, a[0] * a[1] * cc - a[2] * sn,
                              a[0] * a[2] * cc + a[1] * sn, a[1] * a[0] * cc + a[2] * sn,
                              cs + a[1] * a[1] * cc, a[1] * a[2] * cc - a[0] * sn,
                              a[2] * a[0] * cc - a[1] * sn, a[2] * a[1] * cc + a[0] * sn,
                              cs + a[2] * a[2] * cc};
        bool moving = omega != 0.0;
        for (int i = 0; i < 9; ++i) {
            w.qs[i] = qs[i];
            w.q[i] = (i % 4 == 0) ? 1.0 : 0.0;
        }
        for (int d = 0; d < 3; ++d) {
            w.c[d] = c[d];
            w.t[d] = 0.0;
            w.v[d] = v[d];
            w.vdt[d] = v[d] * step;
            w.w[d] = omega * a[d];
            moving = moving || v[d] != 0.0;
        }
        w.type = moving ? type : 0;
        if (mx0.empty()) {
            mx0.assign(3 * size_t(n), 0.0);
            mn0.assign(3 * size_t(n), 0.0);
        }
        if (w.type != 0)
            for (int i = 0; i < n; ++i)
                if (typ[i] == type) {
                    mx0[i] = double(px[i]); mx0[n + i] = double(py[i]); mx0[2 * size_t(n) + i] = double(pz[i]);
                    mn0[i] = double(nx[i]); mn0[n + i] = double(ny[i]); mn0[2 * size_t(n) + i] = double(nz[i]);
                }
        mot[type == OBJ ? 0 : 1] = w;
        return 0;
    }

    bool moving() const { return mot[0].type != 0 || mot[1].type != 0; }

    void move_walls() {
        for (Motion& w : mot) {
            if (w.type == 0) continue;
            double r[9];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    r[3 * i + j] = (w.qs[3 * i] * w.q[j] + w.qs[3 * i + 1] * w.q[3 + j]) +
                                   w.qs[3 * i + 2] * w.q[6 + j];
            for (int i = 0; i < 9; ++i) w.q[i] = r[i];
            for (int d = 0; d < 3; ++d) w.t[d] = w.t[d] + w.vdt[d];
        }
        for (int i = 0; i < n; ++i) {
            const int k = (mot[0].type != 0 && typ[i] == mot[0].type)
                              ? 0 : ((mot[1].type != 0 && typ[i] == mot[1].type) ? 1 : -1);
            if (k < 0) continue;
            const Motion& w = mot[k];
            const double dx = mx0[i] - w.c[0], dy = mx0[n + i] - w.c[1], dz = mx0[2 * size_t(n) + i] - w.c[2];
            const double rx = (w.q[0] * dx + w.q[1] * dy) + w.q[2] * dz;
            const double ry = (w.q[3] * dx + w.q[4] * dy) + w.q[5] * dz;
            const double rz = (w.q[6] * dx + w.q[7] * dy) + w.q[8] * dz;
            const double ax = mn0[i], ay = mn0[n + i], az = mn0[2 * size_t(n) + i];
            px[i] = R((w.c[0] + w.t[0]) + rx);
            py[i] = R((w.c[1] + w.t[1]) + ry);
            pz[i] = R((w.c[2] + w.t[2]) + rz);
            nx[i] = R((w.q[0] * ax + w.q[1] * ay) + w.q[2] * az);
            ny[i] = R((w.q[3] * ax + w.q[4] * ay) + w.q[5] * az);
            nz[i] = R((w.q[6] * ax + w.q[7] * ay) + w.q[8] * az);
            vx[i] = R(w.v[0] + (w.w[1] * rz - w.w[2] * ry));
            vy[i] = R(w.v[1] + (w.w[2] * rx - w.w[0] * rz));
            vz[i] = R(w.v[2] + (w.w[0] * ry - w.w[1] * rx));
        }
    }

    // ---- PrsGrdTrm, corrected-matrix variant (the #if 0 branch, kernel.cu:1435-1648) -------
    // P_min as in the active variant; then the moment matrix sum w r r^T (nine sums, each
    // row a times column b as (w r_a) r_b) and the right side sum w (P_j - P_min) r over the
    // fluid and mirror neighbours inside rp, both scaled by 1/n0_grad; the acceleration is
    // -1/rho M^-1 b through the adjugate over the determinant (kernel.cu:1622-1642). When all
    // nine sums are zero the reference returns without writing d_Acc (kernel.cu:1620), which
    // then still holds the velocity ChkCol stored there (kernel.cu:1275): that is kept.
    void prsgrdtrm_corrected() {
        const R invro = R(-1) / rho;
        const R invn0 = R(1) / n0_grad;
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (typ[i] != FLD) continue;
            R x = px[i], y = py[i], z = pz[i];
            R pmin = prs[i];
            int ix, iy, iz;
            cell3(x, y, z, ix, iy, iz);
            for_fluid(x, y, z, ix, iy, iz, rp, [&](int j) {
                if (j == i || typ[j] != FLD) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rp2) {
                    if (prs[j] < pmin) pmin = prs[j];
                }
            });
            R m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, b[3] = {0, 0, 0};
            int cf = 0, cm = 0;
            auto add = [&](R qx, R qy, R qz, R d2, R pj) {
                R d = std::sqrt(d2);
                R w = wei_grad(d, rp) / d2;
                R wx = w * qx, wy = w * qy, wz = w * qz;
                m[0] = fmar(wx, qx, m[0]); m[1] = fmar(wx, qy, m[1]); m[2] = fmar(wx, qz, m[2]);
                m[3] = fmar(wy, qx, m[3]); m[4] = fmar(wy, qy, m[4]); m[5] = fmar(wy, qz, m[5]);
                m[6] = fmar(wz, qx, m[6]); m[7] = fmar(wz, qy, m[7]); m[8] = fmar(wz, qz, m[8]);
                R wp = w * (pj - pmin);
                b[0] = fmar(wp, qx, b[0]); b[1] = fmar(wp, qy, b[1]); b[2] = fmar(wp, qz, b[2]);
            };
            for_fluid(x, y, z, ix, iy, iz, rp, [&](int j) {
                if (j == i || typ[j] != FLD) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rp2) {
                    add(qx, qy, qz, d2, prs[j]);
                    ++cf;
                }
            });
            for_nb(mstart, mlist, ix, iy, iz, [&](int s) {
                if (s == i) return;  // the slot-index quirk of the active variant (:1575)
                R qx = mx[s] - x, qy = my[s] - y, qz = mz[s] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rp2) {
                    add(qx, qy, qz, d2, mprs[s]);
                    ++cm;
                }
            });
            diag[size_t(i) * D_NCOL + D_GRD_F] = cf;
            diag[size_t(i) * D_NCOL + D_GRD_M] = cm;
            bool zero = true;
            for (int k = 0; k < 9; ++k) {
                m[k] = invn0 * m[k];
                zero = zero && m[k] == R(0);
            }
            if (zero) continue;  // d_Acc keeps ChkCol's velocity
            const R det = R(1) / ((m[0] * m[4] * m[8] + m[1] * m[5] * m[6] + m[2] * m[3] * m[7]) -
                                  (m[2] * m[4] * m[6] + m[0] * m[5] * m[7] + m[1] * m[3] * m[8]));
            const R l0_ = det * (m[4] * m[8] - m[5] * m[7]);
            const R l1_ = det * -(m[1] * m[8] - m[2] * m[7]);
            const R l2_ = det * (m[1] * m[5] - m[2] * m[4]);
            const R l3_ = det * -(m[3] * m[8] - m[5] * m[6]);
            const R l4_ = det * (m[0] * m[8] - m[2] * m[6]);
            const R l5_ = det * -(m[0] * m[5] - m[2] * m[3]);
            const R l6_ = det * (m[3] * m[7] - m[4] * m[6]);
            const R l7_ = det * -(m[0] * m[7] - m[1] * m[6]);
            const R l8_ = det * (m[0] * m[4] - m[1] * m[3]);
            const R r0 = invn0 * b[0], r1 = invn0 * b[1], r2_ = invn0 * b[2];
            ax[i] = invro * (l0_ * r0 + l1_ * r1 + l2_ * r2_);
            ay[i] = invro * (l3_ * r0 + l4_ * r1 + l5_ * r2_);
            az[i] = invro * (l6_ * r0 + l7_ * r1 + l8_ * r2_);
        }
    }

    // ---- PrsGrdTrm, active variant (kernel.cu:1651-1794) ----------------------------------
    void prsgrdtrm() {
        if (grad_mode == 1) {
            prsgrdtrm_corrected();
            return;
        }
        const R invro = R(-1) / rho;
        const R a3 = R(3) / n0_grad;
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            if (typ[i] != FLD) continue;
            R x = px[i], y = py[i], z = pz[i];
            R pmin = prs[i];
            int ix, iy, iz;
            cell3(x, y, z, ix, iy, iz);
            for_fluid(x, y, z, ix, iy, iz, rp, [&](int j) {
                if (j == i || typ[j] != FLD) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rp2) {
                    if (prs[j] < pmin) pmin = prs[j];
                }
            });
            R sx = 0, sy = 0, sz = 0;
            int cf = 0, cm = 0;
            for_fluid(x, y, z, ix, iy, iz, rp, [&](int j) {
                if (j == i || typ[j] != FLD) return;
                R qx = px[j] - x, qy = py[j] - y, qz = pz[j] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rp2) {
                    R d = std::sqrt(d2);
                    R w = wei_grad(d, rp) / d2;
                    R pw = (prs[j] - pmin) * w;
                    sx = fmar(pw, qx, sx); sy = fmar(pw, qy, sy); sz = fmar(pw, qz, sz);
                    ++cf;
                }
            });
            for_nb(mstart, mlist, ix, iy, iz, [&](int s) {
                if (s == i) return;  // the reference compares the mirror slot with i (:1759)
                R qx = mx[s] - x, qy = my[s] - y, qz = mz[s] - z;
                R d2 = dot3(qx, qy, qz, qx, qy, qz);
                if (d2 < rp2) {
                    R d = std::sqrt(d2);
                    R w = wei_grad(d, rp) / d2;
                    R pw = (mprs[s] - pmin) * w;
                    sx = fmar(pw, qx, sx); sy = fmar(pw, qy, sy); sz = fmar(pw, qz, sz);
                    ++cm;
                }
            });
            ax[i] = (invro * sx) * a3;
            ay[i] = (invro * sy) * a3;
            az[i] = (invro * sz) * a3;
            diag[size_t(i) * D_NCOL + D_GRD_F] = cf;
            diag[size_t(i) * D_NCOL + D_GRD_M] = cm;
        }
    }

    // ---- UpPcl2 (kernel.cu:1815-1829) ----------------------------------------------------
    void uppcl2() {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            if (typ[i] == FLD) {
                R a0 = ax[i], a1 = ay[i], a2 = az[i];
                vx[i] = fmar(a0, dt, vx[i]); vy[i] = fmar(a1, dt, vy[i]); vz[i] = fmar(a2, dt, vz[i]);
                px[i] = fmar(a0 * dt, dt, px[i]); py[i] = fmar(a1 * dt, dt, py[i]);
                pz[i] = fmar(a2 * dt, dt, pz[i]);
                ax[i] = ay[i] = az[i] = R(0);
            }
            pav[i] += prs[i];
            chkpcl(i);
        }
    }

    int phase(int ph) {
        switch (ph) {
            case PH_MKBKT: mkbkt(); break;
            case PH_SURFACE_EDGE: surface_edge(); break;
            case PH_RESETMRR: reset_mrr(); break;
            case PH_GENMRR: gen_mrr(); break;
            case PH_MKBKT_MRR: mkbkt_mrr_phase(); break;
            case PH_VSCTRM: vsctrm(); break;
            case PH_UPPCL1: uppcl1(); break;
            case PH_CHKCOL: chkcol(); break;
            case PH_MKPRS: mkprs(); break;
            case PH_PRSGRDTRM: prsgrdtrm(); break;
            case PH_UPPCL2: uppcl2(); break;
            default: return 1;
        }
        return 0;
    }

    // loop body of ClcMPS, kernel.cu:1904-1935
    void step() {
        mkbkt();
        reset_mrr(); gen_mrr(); mkbkt_mrr_phase();
        vsctrm();
        uppcl1();
        mkbkt();
        chkcol();
        mkbkt();  // kernel.cu:1921: same positions, same lists
        mkprs();
        reset_mrr(); gen_mrr(); mkbkt_mrr_phase();
        prsgrdtrm();
        uppcl2();
        if (moving()) {  // walls take their place at the new time, with their edge flags
            move_walls();
            mkbkt();
            surface_edge();
        }
    }
};

struct Any {
    int prec;
    void* p;
};

template <class F> int dispatch(void* h, F&& f) {
    if (!h) return 1;
    Any* a = static_cast<Any*>(h);
    if (a->prec == 0) return f(*static_cast<Oracle<float, float>*>(a->p));
    if (a->prec == 1) return f(*static_cast<Oracle<double, double>*>(a->p));
    return f(*static_cast<Oracle<float, double>*>(a->p));
}

template <class R> void put3(const std::vector<R>& a, const std::vector<R>& b,
                             const std::vector<R>& c, void* out) {
    if (!out) return;
    R* o = static_cast<R*>(out);
    size_t n = a.size();
    std::copy(a.begin(), a.end(), o);
    std::copy(b.begin(), b.end(), o + n);
    std::copy(c.begin(), c.end(), o + 2 * n);
}
template <class R> void get3(std::vector<R>& a, std::vector<R>& b, std::vector<R>& c,
                             const void* in) {
    if (!in) return;
    const R* s = static_cast<const R*>(in);
    size_t n = a.size();
    std::copy(s, s + n, a.begin());
    std::copy(s + n, s + 2 * n, b.begin());
    std::copy(s + 2 * n, s + 3 * n, c.begin());
}

}  // namespace

extern "C" {

void* oracle_create(const oracle_params* p, int32_t n, const int8_t* typ, const void* pos,
                    const void* vel, const void* nrm) {
    if (!p || n < 0 || !typ || !pos || !vel || !nrm) return nullptr;
    Any* a = new Any{p->precision, nullptr};
    if (p->precision == 1) {
        auto* o = new Oracle<double, double>();
        o->init(*p, n, typ, (const double*)pos, (const double*)vel, (const double*)nrm);
        a->p = o;
    } else if (p->precision == 2) {
        auto* o = new Oracle<float, double>();
        o->init(*p, n, typ, (const float*)pos, (const float*)vel, (const float*)nrm);
        a->p = o;
    } else {
        a->prec = 0;
        auto* o = new Oracle<float, float>();
        o->init(*p, n, typ, (const float*)pos, (const float*)vel, (const float*)nrm);
        a->p = o;
    }
    return a;
}

void oracle_destroy(void* h) {
    if (!h) return;
    Any* a = static_cast<Any*>(h);
    if (a->prec == 0) delete static_cast<Oracle<float, float>*>(a->p);
    else if (a->prec == 1) delete static_cast<Oracle<double, double>*>(a->p);
    else delete static_cast<Oracle<float, double>*>(a->p);
    delete a;
}

int oracle_set_threads(int32_t n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int oracle_phase(void* h, int32_t ph) {
    return dispatch(h, [&](auto& o) { return o.phase(ph); });
}

int oracle_set_gradient(void* h, int32_t mode) {
    if (mode < 0 || mode > 1) return 1;
    return dispatch(h, [&](auto& o) {
        o.grad_mode = mode;
        return 0;
    });
}

int oracle_set_wall_motion(void* h, int32_t type, const double* center, const double* axis,
                           double omega, const double* velocity) {
    if (!center || !velocity || (omega != 0.0 && !axis)) return 1;
    return dispatch(h, [&](auto& o) { return o.set_motion(type, center, axis, omega, velocity); });
}

int oracle_step(void* h, int32_t k) {
    return dispatch(h, [&](auto& o) {
        for (int s = 0; s < k; ++s) o.step();
        return 0;
    });
}

int oracle_get_state(void* h, int8_t* typ, void* pos, void* vel, void* acc, void* prs,
                     void* pav) {
    return dispatch(h, [&](auto& o) {
        using R = typename std::remove_reference<decltype(o.px[0])>::type;
        if (typ) std::copy(o.typ.begin(), o.typ.end(), typ);
        put3(o.px, o.py, o.pz, pos);
        put3(o.vx, o.vy, o.vz, vel);
        put3(o.ax, o.ay, o.az, acc);
        if (prs) std::copy(o.prs.begin(), o.prs.end(), static_cast<R*>(prs));
        if (pav) std::copy(o.pav.begin(), o.pav.end(), static_cast<R*>(pav));
        return 0;
    });
}

int oracle_set_state(void* h, const int8_t* typ, const void* pos, const void* vel,
                     const void* acc, const void* prs, const void* pav) {
    return dispatch(h, [&](auto& o) {
        using R = typename std::remove_reference<decltype(o.px[0])>::type;
        if (typ) std::copy(typ, typ + o.n, o.typ.begin());
        get3(o.px, o.py, o.pz, pos);
        get3(o.vx, o.vy, o.vz, vel);
        get3(o.ax, o.ay, o.az, acc);
        if (prs) std::copy(static_cast<const R*>(prs), static_cast<const R*>(prs) + o.n, o.prs.begin());
        if (pav) std::copy(static_cast<const R*>(pav), static_cast<const R*>(pav) + o.n, o.pav.begin());
        // every method of the reference that reads the bucket lists runs after an MkBkt on
        // the same positions, so a replaced state gets fresh lists
        o.mkbkt();
        return 0;
    });
}

int oracle_get_wall_flags(void* h, int8_t* w) {
    return dispatch(h, [&](auto& o) {
        std::copy(o.wse.begin(), o.wse.end(), w);
        return 0;
    });
}

int oracle_set_wall_flags(void* h, const int8_t* w) {
    return dispatch(h, [&](auto& o) {
        std::copy(w, w + o.n, o.wse.begin());
        return 0;
    });
}

int oracle_get_mirrors(void* h, int32_t cap, int32_t* slot, void* pos, void* prs,
                       int32_t* n_out) {
    return dispatch(h, [&](auto& o) {
        using R = typename std::remove_reference<decltype(o.px[0])>::type;
        int k = 0;
        for (size_t s = 0; s < o.mtyp.size(); ++s) {
            if (o.mtyp[s] == GST) continue;
            if (k < cap) {
                if (slot) slot[k] = int32_t(s);
                if (pos) {
                    R* p = static_cast<R*>(pos);
                    p[k] = o.mx[s]; p[cap + k] = o.my[s]; p[2 * size_t(cap) + k] = o.mz[s];
                }
                if (prs) static_cast<R*>(prs)[k] = o.mprs[s];
            }
            ++k;
        }
        if (n_out) *n_out = k;
        return 0;
    });
}

int oracle_set_mirrors(void* h, int32_t nm, const int32_t* slot, const void* pos,
                       const void* prs) {
    return dispatch(h, [&](auto& o) {
        using R = typename std::remove_reference<decltype(o.px[0])>::type;
        o.reset_mrr();
        const R* p = static_cast<const R*>(pos);
        const R* q = static_cast<const R*>(prs);
        for (int k = 0; k < nm; ++k) {
            size_t s = size_t(slot[k]);
            if (s >= o.mtyp.size()) return 1;
            o.mtyp[s] = MRR;
            o.mx[s] = p[k]; o.my[s] = p[nm + k]; o.mz[s] = p[2 * size_t(nm) + k];
            o.mprs[s] = q ? q[k] : R(0);
        }
        o.mkbkt_mrr();
        return 0;
    });
}

int oracle_get_diag(void* h, int32_t* table, void* ndens) {
    return dispatch(h, [&](auto& o) {
        using R = typename std::remove_reference<decltype(o.px[0])>::type;
        for (int i = 0; i < o.n; ++i) {  // bucket index of the current position
            int ix, iy, iz;
            o.diag[size_t(i) * D_NCOL + D_CELL] =
                o.typ[i] == GST ? -1 : o.cell3(o.px[i], o.py[i], o.pz[i], ix, iy, iz);
        }
        if (table) std::copy(o.diag.begin(), o.diag.end(), table);
        if (ndens) std::copy(o.ndens.begin(), o.ndens.end(), static_cast<R*>(ndens));
        return 0;
    });
}

int oracle_get_info(void* h, double* out) {
    return dispatch(h, [&](auto& o) {
        double v[] = {double(o.n0), double(o.lmd), double(o.n0_grad), double(o.lmd_grad),
                      double(o.numn0_grad), double(o.r), double(o.rp), double(o.db),
                      double(o.dbinv), double(o.nbx), double(o.nby), double(o.nbz),
                      double(o.rlim2), double(o.col), double(o.prs_coef), double(o.minc[0]),
                      double(o.minc[1]), double(o.minc[2]), double(o.maxc[0]),
                      double(o.maxc[1]), double(o.maxc[2]), double(o.err_mirror_slot)};
        std::copy(v, v + sizeof(v) / sizeof(v[0]), out);
        return 0;
    });
}

int oracle_get_integrals(void* h, double* out) {
    return dispatch(h, [&](auto& o) {
        double cx = 0, cy = 0, cz = 0, ke = 0, front = -1e300;
        long long cnt = 0;
        for (int i = 0; i < o.n; ++i) {
            if (o.typ[i] != FLD) continue;
            cx += double(o.px[i]); cy += double(o.py[i]); cz += double(o.pz[i]);
            double u = double(o.vx[i]), v = double(o.vy[i]), w = double(o.vz[i]);
            ke += 0.5 * (u * u + v * v + w * w);
            front = std::max(front, double(o.px[i]));
            ++cnt;
        }
        out[0] = cnt ? cx / cnt : 0; out[1] = cnt ? cy / cnt : 0; out[2] = cnt ? cz / cnt : 0;
        out[3] = ke; out[4] = cnt ? front : 0; out[5] = double(cnt);
        return 0;
    });
}

}  // extern "C"
