// mps_adjoint.cuh -- reverse-mode derivative of the explicit MPS step.
//
// The forward step (kernel.cu:1904-1935, as fused in k_pass_a / k_pass_b / k_pass_c) maps
// the fluid state (x, v) to (x', v') through
//   A  S_i = sum_j (v_j - v_i) w(|x_j - x_i|) + sum_m (0 - v_i) w(|m - x_i|),  w = 2 l0 / d^3
//      u_i = v_i + (kn S_i + g) dt,  x*_i = x_i + u_i dt,  u_i <- clamp(u_i)        (r list)
//   B  v**_i = u_i + sum_j c(u_i - u_j, x*_j - x*_i) over fluid, walls, stale mirrors
//      c(du, r) = -(colfac / |r|^2) max(0, du . r) r                             (rlim)
//      n_i = sum_j W(|x*_j - x*_i|) + sum_m W(|m - x*_i|),  W = rp/d - d/rp          (rp)
//      P_i = clamp((n_i - n0) prs_coef rho, 0, Pmax)
//   C  G_i = sum_j (P_j - Pmin_i) f(d) r_ij + mirrors,  f = (rp/d - d/rp) / d^2      (rp)
//      a_i = (invro a3) G_i,  v'_i = clamp(v**_i + a_i dt),  x'_i = x*_i + a_i dt dt
// with mirrors m = H x_owner + const, H = I - nrm nrm^T (nrm recorded per mirror).
//
// The derivative holds every discrete choice of the recorded step fixed: neighbour lists,
// mirror sets, collision branches, the Pmin argmin, clamps and deletions. Neighbour
// relations are symmetric (a pair's squared distance rounds the same from either end), so
// each pair term is gathered by its receiving particle instead of scattered: the kernels
// below read the adjoints of a slot's list neighbours and write only their own slot. Only
// mirror -> owner terms and the Pmin -> argmin term use atomics. Adjoints are double.
#pragma once
#include "mps_kernels.cuh"

namespace mps {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
template <class R> __device__ __forceinline__ D3 d3v(const V4<R>& a) {
    return D3{double(a.x), double(a.y), double(a.z)};
}
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return D3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V4<double> v4(D3 a) { return V4<double>{a.x, a.y, a.z, 0.0}; }
__device__ __forceinline__ D3 d3d(const V4<double>& a) { return D3{a.x, a.y, a.z}; }
__device__ __forceinline__ void atomic_add3(V4<double>* p, D3 a) {
    atomicAdd(&p->x, a.x);
    atomicAdd(&p->y, a.y);
    atomicAdd(&p->z, a.z);
}
// (I - n n^T) a
template <class R> __device__ __forceinline__ D3 reflect_t(const V4<R>& n, D3 a) {
    D3 nn = d3v(n);
    return a - dot(nn, a) * nn;
}
// J^T y of ChkPcl's clamp u -> u umax / |u| (J is symmetric)
__device__ __forceinline__ D3 clamp_t(D3 u, double umax, D3 y) {
    double un = sqrt(dot(u, u));
    D3 h = (1.0 / un) * u;
    return (umax / un) * (y - dot(h, y) * h);
}

// one recorded step: state snapshots in the two slot orders of the step, the neighbour
// lists, and both mirror generations with their reflection normals
template <class R> struct TapeStep {
    // slot order of pass A (bucket order of x)
    int* pid1; V4<R>* x1; V4<R>* v1; V4<R>* up1; int* nA; int* nbA;
    V4<R>* m1pos; int* m1slot; V4<R>* m1nrm; int* mcs1;
    // slot order of passes B and C (bucket order of x*)
    int* pid2; V4<R>* x2; V4<R>* u2; V4<R>* vv2; R* P2; V4<R>* vp2; int* nB; int* nbB;
    V4<R>* m2pos; int* m2slot; V4<R>* m2nrm; int* mcs2;
};

template <class R, class RN> struct AdjArgs {
    const SceneDev<R, RN>* sc;
    int nF, nbK;
    TapeStep<R> t;
    WallView<R> wl;
    // particle-id order (global ids): adjoints of the step's output on entry, of its input
    // on exit; lx_acc collects mirror -> owner terms for x
    V4<double>* lx; V4<double>* lv; V4<double>* lx_acc;
    // slot order of passes B/C
    V4<double>* lG; V4<double>* lvv; V4<double>* lxs; V4<double>* lx_at;
    double* lP; double* lP_at; R* pmin; int* am; int* inv2;
    // particle-id order between the two halves
    V4<double>* lxs_pid; V4<double>* lu_pid;
    // slot order of pass A
    V4<double>* la; V4<double>* lxa; V4<double>* lva;
    double* lkn;  // sum_i S_i . lambda_a_i
    int* err;     // a list longer than its capacity
};

template <class R, class RN>
__device__ __forceinline__ RowCtx<R> adj_row(const SceneDev<R, RN>& sc, const V4<R>& p) {
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    return row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
}

// C1: adjoint of UpPcl2 + ChkPcl for every slot; Pmin and its argmin over the list
template <class R, class RN> __global__ void __launch_bounds__(128) k_adj_c1(AdjArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    const SceneDev<R, RN>& sc = a.sc[0];
    a.lP_at[s] = 0.0;
    a.lx_at[s] = V4<double>{0, 0, 0, 0};
    const V4<R> pre = a.t.vp2[s];
    const int st = int(pre.w);
    const int pid = a.t.pid2[s];
    a.inv2[pid] = s;
    const V4<double> zero{0, 0, 0, 0};
    R pm = R(0);
    int am = -1;
    if (st != kTapeDead) {
        const int n = a.t.nB[s];
        if (n > a.nbK) {
            atomicAdd(a.err, 1);
        } else {
            const V4<R> p = a.t.x2[s];
            pm = a.t.P2[s];
            for (int k = 0; k < n; ++k) {
                const int j = a.t.nbB[list_at(s, k, a.nbK)];
                const V4<R> q = ldg4(a.t.x2 + j);
                R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
                if (dot3(dx, dy, dz, dx, dy, dz) < sc.rp2) {
                    R pj = __ldg(a.t.P2 + j);
                    if (pj < pm) { pm = pj; am = j; }
                }
            }
        }
    }
    a.pmin[s] = pm;
    a.am[s] = am;
    if (st == kTapeDead || st == kTapeDeleted) {
        a.lG[s] = zero; a.lvv[s] = zero; a.lxs[s] = zero;
        return;
    }
    const double dt = double(sc.dt);
    const D3 lxo = d3d(a.lx[pid]), lvo = d3d(a.lv[pid]);
    const D3 lu = st == kTapeClamped ? clamp_t(d3v(pre), double(sc.umax), lvo) : lvo;
    const D3 la = dt * lu + (dt * dt) * lxo;
    a.lG[s] = v4((double(sc.invro) * double(sc.a3)) * la);
    a.lvv[s] = v4(lu);
    a.lxs[s] = v4(lxo);
}

// pressure-gradient pair factor f(d) = (rp/d - d/rp) / d^2 and (df/dd) / d
__device__ __forceinline__ void grad_f(double d2, double rp, double& f, double& fp) {
    double d = sqrt(d2);
    f = (rp / d - d / rp) / d2;
    fp = (-3.0 * rp / (d2 * d2) + 1.0 / (rp * d2)) / d;
}

// C2: adjoint of PrsGrdTrm, gathered per slot
template <class R, class RN> __global__ void __launch_bounds__(128) k_adj_c2(AdjArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    const SceneDev<R, RN>& sc = a.sc[0];
    const int st = int(a.t.vp2[s].w);
    const int n = a.t.nB[s];
    if (st == kTapeDead || n > a.nbK) {
        a.lP[s] = 0.0;
        return;
    }
    const V4<R> p = a.t.x2[s];
    const D3 x = d3v(p);
    const double Ps = double(a.t.P2[s]), pms = double(a.pmin[s]), rp = double(sc.rp);
    const D3 lGs = d3d(a.lG[s]);
    D3 accx = d3d(a.lxs[s]), sphi = d3(0, 0, 0);
    double accP = 0.0;
    for (int k = 0; k < n; ++k) {
        const int i = a.t.nbB[list_at(s, k, a.nbK)];
        const V4<R> q = ldg4(a.t.x2 + i);
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        if (!(dot3(dx, dy, dz, dx, dy, dz) < sc.rp2)) continue;
        const D3 r = d3v(q) - x;
        double f, fp;
        grad_f(dot(r, r), rp, f, fp);
        const D3 lGi = d3d(a.lG[i]);
        // G_i holds (P_s - Pmin_i) phi(x_s - x_i), G_s holds (P_i - Pmin_s) phi(r)
        const D3 y = (Ps - double(a.pmin[i])) * lGi - (double(a.t.P2[i]) - pms) * lGs;
        accx = accx + f * y + (fp * dot(r, y)) * r;
        accP -= f * dot(r, lGi);
        sphi = sphi + f * r;
    }
    // mirrors of the second generation (the reference skips the slot equal to i, :1759)
    const RowCtx<R> c = adj_row(sc, p);
    const int skip_slot = (a.t.pid2[s] - sc.pbase) + kNumMRR * sc.pbase;
    for_rows(sc, a.t.mcs2, c, sc.skip_rp, [&](int k) {
        const int slot = __ldg(a.t.m2slot + k);
        if (slot == skip_slot) return;
        const V4<R> q = ldg4(a.t.m2pos + k);
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        if (!(dot3(dx, dy, dz, dx, dy, dz) < sc.rp2)) return;
        const D3 r = d3v(q) - x;
        double f, fp;
        grad_f(dot(r, r), rp, f, fp);
        sphi = sphi + f * r;
        const int os = a.inv2[slot / kNumMRR];
        atomicAdd(a.lP_at + os, f * dot(r, lGs));
        const D3 lm = (double(q.w) - pms) * (f * lGs + (fp * dot(r, lGs)) * r);
        accx = accx - lm;
        atomic_add3(a.lx_at + os, reflect_t(a.t.m2nrm[k], lm));
    });
    const double lpmin = -dot(sphi, lGs);
    if (a.am[s] < 0) accP += lpmin;
    else atomicAdd(a.lP_at + a.am[s], lpmin);
    a.lxs[s] = v4(accx);
    a.lP[s] = accP;
}

// lambda of the number density of slot s (EOS, kernel.cu:1388-1406)
template <class R, class RN>
__device__ __forceinline__ double adj_ln(const AdjArgs<R, RN>& a, const SceneDev<R, RN>& sc, int s) {
    const double P = double(a.t.P2[s]);
    if (!(P > 0.0 && P < double(sc.pmax))) return 0.0;
    return double(sc.prs_coef) * double(sc.rho) * (a.lP[s] + a.lP_at[s]);
}

// collision term of pair (s, j) with r = x_j - x*_s and du = u_s - u_j: adds the u_s part
// of the adjoint to accu and returns the x*_s part. y = lambda_j - lambda_s for a fluid
// pair (both ends gathered at once), -lambda_s for a wall or a mirror (whose r-derivative
// is minus the returned vector).
__device__ __forceinline__ D3 col_adj(double colfac, D3 r, double d2, D3 du, D3 y, D3& accu) {
    const double f = dot(du, r);
    if (!(f > 0.0)) return d3(0, 0, 0);
    const double al = colfac / d2, ry = dot(r, y);
    accu = accu + (al * ry) * r;
    return (-al * f) * y + (-al * ry) * du + (2.0 * al * f * ry / d2) * r;
}

// B2: adjoint of ChkCol + MkPrs, gathered per slot; writes the adjoints of x* and u in
// particle-id order
template <class R, class RN> __global__ void __launch_bounds__(128) k_adj_b2(AdjArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    const SceneDev<R, RN>& sc = a.sc[0];
    const int st = int(a.t.vp2[s].w);
    const int pid = a.t.pid2[s];
    const int n = a.t.nB[s];
    if (st == kTapeDead || n > a.nbK) {
        a.lxs_pid[pid] = V4<double>{0, 0, 0, 0};
        a.lu_pid[pid] = V4<double>{0, 0, 0, 0};
        return;
    }
    const V4<R> p = a.t.x2[s];
    const D3 x = d3v(p), u = d3v(a.t.u2[s]);
    const D3 lvs = d3d(a.lvv[s]);
    const double lns = adj_ln(a, sc, s), rp = double(sc.rp), colfac = double(sc.colfac);
    D3 accx = d3d(a.lxs[s]) + d3d(a.lx_at[s]), accu = lvs;
    for (int k = 0; k < n; ++k) {
        const int i = a.t.nbB[list_at(s, k, a.nbK)];
        const V4<R> q = ldg4(a.t.x2 + i);
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        const R d2r = dot3(dx, dy, dz, dx, dy, dz);
        const D3 r = d3v(q) - x;
        const double d2 = dot(r, r);
        if (d2r <= sc.rp_lt) {  // both densities: n_s and n_i hold W(|r|)
            const double d = sqrt(d2);
            const double wp = (-rp / d2 - 1.0 / rp) / d;  // W'(d) / d
            accx = accx - (wp * (lns + adj_ln(a, sc, i))) * r;
        }
        if (d2r < sc.rlim2)
            accx = accx + col_adj(colfac, r, d2, u - d3v(a.t.u2[i]), d3d(a.lvv[i]) - lvs, accu);
    }
    const RowCtx<R> c = adj_row(sc, p);
    const D3 mlvs = d3(-lvs.x, -lvs.y, -lvs.z);
    for_rows(sc, a.wl.cs, c, sc.skip_rw, [&](int j) {
        const V4<R> q = ldg4(a.wl.pos + j);
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        if (!(dot3(dx, dy, dz, dx, dy, dz) < sc.rlimw2)) return;
        const D3 r = d3v(q) - x;
        accx = accx + col_adj(colfac, r, dot(r, r), u - d3v(ldg4(a.wl.vel + j)), mlvs, accu);
    });
    // the step's first mirror generation (built from x, not x*: kernel.cu:1904-1921)
    for_rows(sc, a.t.mcs1, c, sc.skip_rc, [&](int k) {
        const V4<R> q = ldg4(a.t.m1pos + k);
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        const R d2r = dot3(dx, dy, dz, dx, dy, dz);
        const bool col = d2r < sc.rlim2, dens = d2r <= sc.rp_lt;
        if (!col && !dens) return;
        const D3 r = d3v(q) - x;
        const double d2 = dot(r, r);
        // every term depends on r = m - x*: x* receives gx, the mirror's owner -H gx
        D3 gx = d3(0, 0, 0);
        if (col) gx = col_adj(colfac, r, d2, u, mlvs, accu);
        if (dens && lns != 0.0) {
            const double d = sqrt(d2);
            const double wp = (-rp / d2 - 1.0 / rp) / d;
            gx = gx - (wp * lns) * r;
        }
        if (gx.x != 0.0 || gx.y != 0.0 || gx.z != 0.0) {
            accx = accx + gx;
            atomic_add3(a.lx_acc + __ldg(a.t.m1slot + k) / kNumMRR,
                        reflect_t(a.t.m1nrm[k], d3(-gx.x, -gx.y, -gx.z)));
        }
    });
    a.lxs_pid[pid] = v4(accx);
    a.lu_pid[pid] = v4(accu);
}

// A1: adjoint of UpPcl1 + ChkPcl for every slot of pass A
template <class R, class RN> __global__ void __launch_bounds__(128) k_adj_a1(AdjArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    const SceneDev<R, RN>& sc = a.sc[0];
    const V4<R> pre = a.t.up1[s];
    const int st = int(pre.w);
    const V4<double> zero{0, 0, 0, 0};
    if (st == kTapeDead || st == kTapeDeleted) {
        a.la[s] = zero; a.lxa[s] = zero; a.lva[s] = zero;
        return;
    }
    const int pid = a.t.pid1[s];
    const double dt = double(sc.dt);
    const D3 lx = d3d(a.lxs_pid[pid]);
    D3 lu = d3d(a.lu_pid[pid]);
    if (st == kTapeClamped) lu = clamp_t(d3v(pre), double(sc.umax), lu);
    const D3 lup = lu + dt * lx;  // x* was advanced with the velocity before the clamp
    a.la[s] = v4(dt * lup);
    a.lxa[s] = v4(lx);
    a.lva[s] = v4(lup);
}

// A2: adjoint of VscTrm, gathered per slot; writes the adjoints of the step's input in
// particle-id order and accumulates sum S . lambda_a for the viscosity
template <class R, class RN> __global__ void __launch_bounds__(128) k_adj_a2(AdjArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double part = 0.0;
    if (s < a.nF) {
        const SceneDev<R, RN>& sc = a.sc[0];
        const int st = int(a.t.up1[s].w);
        const int pid = a.t.pid1[s];
        const int n = a.t.nA[s];
        if (st == kTapeDead || n > a.nbK) {
            if (n > a.nbK && st != kTapeDead) atomicAdd(a.err, 1);
            a.lx[pid] = V4<double>{0, 0, 0, 0};
            a.lv[pid] = V4<double>{0, 0, 0, 0};
        } else {
            const V4<R> p = a.t.x1[s];
            const D3 x = d3v(p), v = d3v(a.t.v1[s]);
            const double kn = double(sc.kn), two_l0 = double(sc.two_l0);
            const D3 las = d3d(a.la[s]);
            const D3 lSs = kn * las;
            D3 accx = d3d(a.lxa[s]), accv = d3d(a.lva[s]), S = d3(0, 0, 0);
            for (int k = 0; k < n; ++k) {
                const int i = a.t.nbA[list_at(s, k, a.nbK)];
                const D3 r = d3v(ldg4(a.t.x1 + i)) - x;
                const D3 vi = d3v(ldg4(a.t.v1 + i));
                const double d2 = dot(r, r), d = sqrt(d2), w = two_l0 / (d2 * d);
                S = S + w * (vi - v);
                // S_i holds (v_s - v_i) w, S_s holds (v_i - v_s) w; grad w(x_s - x_i) = 3 w r / d^2
                const D3 y = kn * d3d(a.la[i]) - lSs;
                accv = accv + w * y;
                accx = accx + ((3.0 * w / d2) * dot(v - vi, y)) * r;
            }
            const RowCtx<R> c = adj_row(sc, p);
            const double vl = dot(v, lSs);
            for_rows(sc, a.t.mcs1, c, sc.skip_r, [&](int k) {
                const V4<R> q = ldg4(a.t.m1pos + k);
                R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
                if (!(dot3(dx, dy, dz, dx, dy, dz) <= sc.r_le)) return;
                const D3 r = d3v(q) - x;
                const double d2 = dot(r, r), d = sqrt(d2), w = two_l0 / (d2 * d);
                S = S - w * v;
                accv = accv - w * lSs;
                const D3 gm = ((3.0 * w / d2) * vl) * r;  // d/dm of -(v . lambda_S) w(|m - x|)
                accx = accx - gm;
                atomic_add3(a.lx_acc + __ldg(a.t.m1slot + k) / kNumMRR, reflect_t(a.t.m1nrm[k], gm));
            });
            part = dot(S, las);
            a.lx[pid] = v4(accx);
            a.lv[pid] = v4(accv);
        }
    }
    // block sum of S . lambda_a, one atomic per block
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    __shared__ double wsum[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wsum[w] = part;
    __syncthreads();
    if (w == 0) {
        part = lane < int(blockDim.x >> 5) ? wsum[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
        if (lane == 0 && part != 0.0) atomicAdd(a.lkn, part);
    }
}

// fold the mirror -> owner terms into the adjoint of x and clear them for the next step
static __global__ void k_adj_fin(const int* __restrict__ ids, int n, V4<double>* lx,
                                 V4<double>* lx_acc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int pid = ids[k];
    const V4<double> a = lx[pid], b = lx_acc[pid];
    lx[pid] = V4<double>{a.x + b.x, a.y + b.y, a.z + b.z, 0.0};
    lx_acc[pid] = V4<double>{0, 0, 0, 0};
}

// SoA double (x[n], y[n], z[n]) <-> V4<double> in particle-id order
static __global__ void k_adj_in(const double* __restrict__ src, int n, V4<double>* dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    dst[k] = V4<double>{src[k], src[n + k], src[2 * size_t(n) + k], 0.0};
}
// dst[pid] = src[pid] for the fluid particle ids
static __global__ void k_adj_pick(const int* __restrict__ ids, int n, const V4<double>* src,
                                  V4<double>* dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    dst[ids[k]] = src[ids[k]];
}
static __global__ void k_adj_out(const V4<double>* __restrict__ src, int n, double* dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const V4<double> v = src[k];
    dst[k] = v.x;
    dst[n + k] = v.y;
    dst[2 * size_t(n) + k] = v.z;
}

}  // namespace mps
