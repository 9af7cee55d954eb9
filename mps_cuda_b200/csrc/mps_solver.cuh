// mps_solver.cuh -- host side of the B200 MPS solver (templated on the arithmetic).
//
// One handle owns the device state of one or more scenes. The reference keeps that state
// in public members of `class MPS` (class.cuh:49-141) and drives it from ClcMPS
// (kernel.cu:1872-1943) with a blocking cudaDeviceSynchronize after every kernel; here the
// whole step is queued on one stream (optionally replayed as a CUDA graph) and nothing
// synchronises until the caller reads data back.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mps_b200.h"
#include "mps_adjoint.cuh"
#include "mps_kernels.cuh"

namespace mps {

extern thread_local std::string g_last_error;

struct ApiError : std::runtime_error {
    int code;
    ApiError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            throw ApiError(e_ == cudaErrorMemoryAllocation ? MPS_ERR_NOMEM : MPS_ERR_CUDA,   \
                           std::string(#call) + ": " + cudaGetErrorString(e_));              \
        }                                                                                    \
    } while (0)

#define CKL() CK(cudaGetLastError())
// after a kernel launch inside the solver: count it and check the launch
#define KL()                          \
    do {                              \
        ++launches;                   \
        CK(cudaGetLastError());       \
    } while (0)

// ---- derived constants (AlcBkt + SetPara, kernel.cu:307-415) ----------------------------
// Grid limits: fine cells (27 per bucket, plus the cell of unlisted particles and the end
// of the start table) are indexed by int32 across all scenes of a handle.
constexpr long long kMaxBucketsPerAxis = 1LL << 20;
constexpr long long kMaxFineCells = (1LL << 31) - 2;

template <class R> static R wei(R d, R re) { return ((re / d) + (d / re)) - R(2); }
template <class R> static R wei_grad_h(R d, R re) { return (re / d) - (d / re); }

// largest t with sqrt(t) <= r (le = true) or sqrt(t) < r (le = false), so that
// `sqrt(d2) <= r` can be tested as `d2 <= t` without a square root
template <class R> static R sqrt_threshold(R r, bool le) {
    auto ok = [&](R t) { R s = std::sqrt(t); return le ? (s <= r) : (s < r); };
    R t = r * r;
    while (!ok(t)) t = std::nextafter(t, R(0));
    for (;;) {
        R u = std::nextafter(t, R(INFINITY));
        if (!ok(u)) break;
        t = u;
    }
    return t;
}

template <class R, class RN>
static void derive_scene(const mps_params& p, int cbase, int fbase, int pbase, int pcount,
                         SceneDev<R, RN>& s, mps_info& inf) {
    std::memset(&s, 0, sizeof(s));
    const R l0 = R(p.pcl_dst);
    R maxc[3];
    for (int d = 0; d < 3; ++d) {
        s.minc[d] = R(double(R(p.min[d])) - 3.1 * double(l0));  // kernel.cu:26-31
        maxc[d] = R(double(R(p.max[d])) + 3.1 * double(l0));
        s.g[d] = R(p.g[d]);
    }
    const R r = l0 * R(3.1), r2 = r * r, rp = l0 * R(2.1), rp2 = rp * rp;
    const R db = l0 * R(3.1), dbinv = R(1) / db;
    s.db = db;
    s.dbinv = dbinv;
    // kernel.cu:317-319. The extents are checked before any int conversion, and the bucket
    // count in 64 bits, so that no grid too large for the int32 cell indices of the bucket
    // builds (27 fine cells per bucket, plus the unlisted cell) wraps to a small value.
    long long nbl[3];
    for (int d = 0; d < 3; ++d) {
        const R t = (maxc[d] - s.minc[d]) * dbinv;
        if (!(t >= R(0) && t < R(kMaxBucketsPerAxis)))
            throw ApiError(MPS_ERR_OVERFLOW, "the bucket grid has more than " +
                                                 std::to_string(kMaxBucketsPerAxis) +
                                                 " buckets along an axis");
        nbl[d] = (long long)(t) + 3;
    }
    const long long nbxyz = nbl[0] * nbl[1] * nbl[2];
    if (27 * nbxyz + 2 > kMaxFineCells)
        throw ApiError(MPS_ERR_OVERFLOW, "the bucket grid needs " + std::to_string(nbxyz) +
                                             " buckets, more than int32 fine-cell indices hold");
    s.nbx = int(nbl[0]);
    s.nby = int(nbl[1]);
    s.nbz = int(nbl[2]);
    s.nbxy = s.nbx * s.nby;
    s.cbase = cbase;
    s.pbase = pbase;
    s.pcount = pcount;
    s.fbase = fbase;
    s.ihf = float(3.0 * double(dbinv));  // fine cell f spans t in [(f - 3) / 3, (f - 2) / 3)
    s.hf = float(1.0 / (3.0 * double(dbinv)));
    // lattice sums, kernel.cu:336-366
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
                    tn0g += wei_grad_h(d, rp);
                    tlg += d2 * wei_grad_h(d, rp);
                    cnt += 1;
                }
                if (d2 < r2) {
                    tn0 += wei(d, r);
                    tl += d2 * wei(d, r);
                }
            }
    const R n0 = tn0, n0_grad = tn0g;
    const R rlim = l0 * R(p.dst_lmt_rat), rlim2 = rlim * rlim;  // kernel.cu:370-371
    const R col = R(p.col_rat) + R(1);                           // kernel.cu:373
    const R rho = R(p.rho), knm = R(p.knm_vsc), snd = R(p.snd);
    const R rw = R(0.45) * l0;  // kernel.cu:1184
    s.r = r; s.r2 = r2; s.r_le = sqrt_threshold(r, true);
    s.rp = rp; s.rp2 = rp2; s.rp_lt = sqrt_threshold(rp, false);
    s.rlim2 = rlim2;
    // one list serves dist2 < rlim2 (ChkCol), sqrt(dist2) < rp (MkPrs), dist2 < rp2 (PrsGrdTrm)
    s.list_thr = std::max({std::nextafter(rlim2, R(0)), s.rp_lt, std::nextafter(rp2, R(0))});
    s.rlimw2 = rw * rw;
    s.edge_r2 = (R(1) * l0) * (R(1) * l0);
    s.wall_dist0 = R(10) * r;
    s.two_l0 = R(2) * l0;
    s.kn = (R(1) / n0) * knm;
    s.dt = R(p.dt);
    s.umax = R(p.umax);
    for (int d = 0; d < 3; ++d) {
        R t = R(3.1) * l0;
        s.lo[d] = s.minc[d] + t;
        s.hi[d] = maxc[d] - t;
    }
    s.colfac = (col * rho) / (rho + rho);
    s.invro = R(-1) / rho;
    s.a3 = R(3) / n0_grad;
    s.invn0g = R(1) / n0_grad;
    const double m = 1e-3 * double(db);
    auto sq = [&](double v) { return R((v + m) * (v + m)); };
    s.skip_r = sq(double(r));
    s.skip_rp = sq(double(rp));
    s.skip_rl = sq(double(rlim));
    s.skip_rw = sq(double(rw));
    s.skip_rc = sq(std::max(double(rlim), double(rp)));
    // number density / EOS arithmetic
    RN n0g;
    if (sizeof(RN) == sizeof(R)) {
        n0g = RN(n0_grad);
    } else {
        RN acc = 0, l0n = RN(l0), rpn = RN(rp), rp2n = rpn * rpn;
        for (int ix = -10; ix < 10; ++ix)
            for (int iy = -10; iy < 10; ++iy)
                for (int iz = -10; iz < 10; ++iz) {
                    RN x = l0n * RN(ix), y = l0n * RN(iy), z = l0n * RN(iz);
                    RN d2 = x * x + y * y + z * z;
                    if (d2 == RN(0)) continue;
                    if (d2 < rp2n) acc += wei_grad_h(RN(std::sqrt(d2)), rpn);
                }
        n0g = acc;
    }
    s.n0g = n0g;
    s.prs_coef = RN(snd) * RN(snd) / n0g;  // kernel.cu:409
    s.pmax = RN(R(p.pmax));
    s.rho = RN(rho);
    s.rp_n = RN(rp);

    std::memset(&inf, 0, sizeof(inf));
    inf.nbx = s.nbx; inf.nby = s.nby; inf.nbz = s.nbz; inf.nbxyz = s.nbxy * s.nbz;
    inf.r = r; inf.rp = rp; inf.db = db; inf.dbinv = dbinv;
    inf.n0 = n0; inf.lmd = tl / tn0; inf.n0_grad = n0_grad; inf.lmd_grad = tlg / tn0g;
    inf.numn0_grad = cnt;
    inf.rlim2 = rlim2; inf.col = col; inf.prs_coef = double(s.prs_coef); inf.pmax = double(s.pmax);
    inf.umax = s.umax; inf.dt = s.dt; inf.snd = snd;
    for (int d = 0; d < 3; ++d) { inf.minc[d] = s.minc[d]; inf.maxc[d] = maxc[d]; }
}

// ---- device allocation ---------------------------------------------------------------------
struct DevArena {
    std::vector<void*> ptrs;
    template <class T> T* get(size_t n) {
        void* p = nullptr;
        size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw ApiError(MPS_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~DevArena() {
        for (void* p : ptrs) cudaFree(p);
    }
};

template <class R> struct FluidBuf {
    V4<R>* pos; V4<R>* vel; V4<R>* acc; R* prs; R* pav; int* pid; int8_t* typ;
};
template <class R> struct MirrorBuf {
    V4<R>* pos; int* slot;
};

// The motion of one wall type: the step's rotation by omega * dt about the unit axis
// (Rodrigues' formula), the step's translation v * dt, and q = identity, t = 0.
inline WallMotion wall_motion(int type, const double* c, const double* axis, double omega,
                              const double* v, double dt) {
    WallMotion w{};
    double a[3] = {0.0, 0.0, 1.0};
    if (omega != 0.0) {
        const double nn = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
        if (!(nn > 0.0) || !std::isfinite(nn))
            throw ApiError(MPS_ERR_ARG, "the rotation axis must be a non-zero finite vector");
        for (int d = 0; d < 3; ++d) a[d] = axis[d] / nn;
    }
    const double th = omega * dt, cs = std::cos(th), sn = std::sin(th), cc = 1.0 - cs;
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
        w.vdt[d] = v[d] * dt;
        w.w[d] = omega * a[d];
        moving = moving || v[d] != 0.0;
    }
    w.type = moving ? type : 0;
    return w;
}

struct SolverBase {
    virtual ~SolverBase() {}
    int dev = 0;
    cudaStream_t stream = 0, own_stream = 0;
    int nscene = 0, nT = 0, nF = 0, nW = 0, C = 0, CF = 0, cap = 0;
    int precision = 0;
    std::vector<mps_info> infos;
    std::vector<int> counts;
    bool diag_on = false, graph_on = false;
    int skip_opt = 1, block = 128;
    int grad_mode = MPS_GRAD_STANDARD;  // PrsGrdTrm variant (MPS_OPT_GRADIENT)
    int stage_mode = MPS_STAGE_GLOBAL;  // pass A's candidate source (MPS_OPT_STAGING)
    int stage_cap = 0;                  // candidates staged per block (MPS_OPT_STAGE_CAPACITY)
    int batch_a = 4;                    // VscTrm's candidates in flight (MPS_OPT_CANDIDATE_BATCH)
    int reg_bound = 0;                  // passes B, C, A at their alternate register bound (bits 0-2)
    int overlap = 3;                    // work on a second stream (MPS_OPT_OVERLAP bits 0-1)
    long long steps = 0;
    long long launches = 0;       // kernels launched (graph replays included)
    long long head_launches = 0;  // kernels of one captured step up to PrsGrdTrm
    long long tail_launches = 0;  // kernels of one captured step end (mirrors, bucket builds)
    bool timing_on = false;
    double t_ms[MPS_K_COUNT] = {};
    long long t_n[MPS_K_COUNT] = {};
    int blk[MPS_K_COUNT] = {128, 128, 128, 128, 256, 256};  // threads per block per group
    virtual void timing(int k, double* ms, long long* n, bool reset) = 0;
    virtual void autotune(int trial, int32_t* chosen) = 0;
    virtual void step(int n) = 0;
    virtual void phase(int ph) = 0;
    virtual void get_state(int8_t*, void*, void*, void*, void*, void*) = 0;
    virtual void set_state(const int8_t*, const void*, const void*, const void*, const void*,
                           const void*) = 0;
    virtual void get_wall_flags(int8_t*) = 0;
    virtual int get_mirrors(int which, int cap, int32_t* slot, void* pos, void* prs) = 0;
    virtual void get_diag(int32_t* table, void* ndens) = 0;
    virtual void get_counters(mps_counters*) = 0;
    virtual void get_work(mps_work*) = 0;
    virtual void integrals(int scene, double out[6]) = 0;
    virtual void invalidate_graph() = 0;
    virtual void set_list_capacity(int k) = 0;  // 0: the full capacity
    virtual int list_capacity() const = 0;
    // WrtDat's snapshot into device staging (id order, state type) and the second mirror
    // generation; the mirror count goes to pinned host memory. Then pav = 0 (kernel.cu:289).
    virtual void output_snapshot(void* pos, void* vel, void* prs, void* pav, int8_t* typ,
                                 void* mpos, int* mslot, int* mcount_host) = 0;
    virtual void get_wall_normals(void* nrm) = 0;  // inward normals, SoA, id order
    virtual void set_wall_motion(int type, const double* c, const double* axis, double omega,
                                 const double* v) = 0;
    virtual void adjoint_record(int nsteps, int every) = 0;
    virtual void adjoint_backward(const double* lam_pos, const double* lam_vel, double* g_pos,
                                  double* g_vel, double* g_nu) = 0;
};

}  // namespace mps

// the C-ABI's opaque handle: one solver (of one or more scenes)
struct mps_handle {
    std::unique_ptr<mps::SolverBase> s;
};

namespace mps {

// Choices of the autotuner, kept per (precision, batched, log2 of the fluid count) for the
// life of the process: a handle created later in the same class starts from them.
struct TuneKey {
    int precision, batched, size_class;
    bool operator<(const TuneKey& o) const {
        if (precision != o.precision) return precision < o.precision;
        if (batched != o.batched) return batched < o.batched;
        return size_class < o.size_class;
    }
};
struct Tuned {
    int blk[MPS_K_COUNT];
    int stage, batch, regb;
};
bool tuned_cache_get(const TuneKey& k, Tuned* out);
void tuned_cache_put(const TuneKey& k, const Tuned& t);

template <class R, class RN> class Solver final : public SolverBase {
   public:
    using SD = SceneDev<R, RN>;
    DevArena ar;
    std::vector<SD> hsc;
    SD* d_sc = nullptr;
    int* d_nbxyz = nullptr;
    FluidBuf<R> S, S2;
    V4<R>* t_pos; V4<R>* t_vel; R* t_prs; int8_t* t_typ;
    // walls, sorted once
    V4<R>* w_pos; V4<R>* w_nrm; V4<R>* w_vel; int* w_id; int8_t* w_typ; int8_t* w_se;
    int* wcs;
    // walls in load order (the bucket build's source), and the moving walls' motion
    V4<R>* tw_pos = nullptr; V4<R>* tw_vel = nullptr; V4<R>* tw_nrm = nullptr;
    int8_t* tw_typ = nullptr; int* tw_id = nullptr;
    double *mx0 = nullptr, *mn0 = nullptr;  // reference state of the moving walls
    WallMotion* d_motion = nullptr;
    WallMotion hmot[2] = {};
    bool motion_on = false;
    // mirrors: raw list U and two sorted generations
    MirrorBuf<R> U, M1, M2;
    int *mcs1, *mcs2;
    int* cs;
    // fluid positions in row-major fine-cell order (slot in w) and that order's cell starts
    V4<R>* posf;
    int *csr, *count_f;
    // the fluid build's start tables by bucket rows (k_fine_rows_*): per bucket row and per
    // fine row totals, then starts; per scene the bucket rows before it
    int *row_tot, *frow_tot, *row_scan;
    int nrows = 0;
    int row_threads = 256;  // threads per bucket row block: the longest row rounded up
    bool posf_stale = false;  // particles moved in place since the copy was made
    // bucket-build scratch
    int *key, *rnk, *seg, *count, *part;
    int* d_fluid_ids;
    int* d_wall_ids;
    int* d_nF;
    DevCounters* cnt;
    int32_t* diag;
    RN* ndens;
    IdState<R> io;
    double* d_integ;
    int* nb;
    int* nbcnt;
    int8_t* near_wall;
    int8_t *near_m1, *near_m2;  // near flags of the mirror tables M1 / M2 (k_near_wall on mcs)
    static constexpr int kListCap = 160;  // about 125 neighbours lie inside r at rest density
    int nbK = kListCap;                    // list capacity in use (MPS_OPT_LIST_CAPACITY)
    std::vector<int> fluid_ids, wall_ids;
    bool lists_valid = false, sorted = false, m1_valid = false, acc_dirty = false;
    // Captured graphs of a step's body (passes A to C, moving walls) and of a step's end (the
    // next step's mirrors and bucket builds), one per buffer the sorted state starts in: each
    // holds one fluid bucket build, which moves the state from S to S2, so a graph's baked
    // pointers fit only the buffer it was captured from. A replay swaps S and S2 on the host
    // as the captured build did.
    cudaGraphExec_t gx_head[2] = {nullptr, nullptr};
    cudaGraphExec_t gx_tail[2] = {nullptr, nullptr};
    int swaps_head = 0, swaps_tail = 0;  // fluid bucket builds in each
    const void* sbuf0 = nullptr;          // S.pos at allocation: buffer 0
    int swap_count = 0;                   // fluid bucket builds issued on the host
    bool gexec_diag = false;
    // The end of the latest step (the next step's first mirror generation and the bucket
    // build of x^{n+1}) has not run yet: the state lives in the scratch arrays t_* in the
    // slot order of S. It runs when the next step starts or when something reads the sorted
    // state, so a state replaced in between (mps_set_state) wastes no build.
    bool tail_pending = false;
    // the handle's second stream (MPS_OPT_OVERLAP), created with the handle, at the device's
    // highest priority: the work forked to it (the step end's fluid bucket build, the second
    // mirror generation) gets SMs while the main stream's long kernel has blocks pending;
    // the fork and join events
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void ensure_side() {
        if (side) return;
        int lo = 0, hi = 0;
        CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        CK(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, hi));
    }
    // launches issued in its scope go to stream `to`; the handle's stream is restored on exit
    struct OnStream {
        Solver* s;
        cudaStream_t prev;
        OnStream(Solver* s_, cudaStream_t to) : s(s_), prev(s_->stream) { s->stream = to; }
        ~OnStream() { s->stream = prev; }
    };
    // CUDA events bracketing kernel groups when timing_on
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
    cudaEvent_t ev_get() {
        if (ev_pool.empty()) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            return e;
        }
        cudaEvent_t e = ev_pool.back();
        ev_pool.pop_back();
        return e;
    }
    struct Scope {
        Solver* s;
        int k;
        cudaEvent_t a = nullptr;
        Scope(Solver* s_, int k_) : s(s_), k(k_) {
            if (s->timing_on) {
                a = s->ev_get();
                CK(cudaEventRecord(a, s->stream));
            }
        }
        ~Scope() {
            if (!a) return;
            cudaEvent_t b = nullptr;
            if (!s->ev_pool.empty()) {
                b = s->ev_pool.back();
                s->ev_pool.pop_back();
            } else if (cudaEventCreate(&b) != cudaSuccess) {
                b = nullptr;
            }
            if (b && cudaEventRecord(b, s->stream) == cudaSuccess) {
                s->ev_pending.push_back({k, {a, b}});
            } else {  // timing of this group is lost; the error surfaces at the next check
                s->ev_pool.push_back(a);
                if (b) s->ev_pool.push_back(b);
            }
        }
    };
    void timing(int k, double* ms, long long* n, bool reset) override {
        CK(cudaStreamSynchronize(stream));
        for (auto& pe : ev_pending) {
            float x = 0;
            CK(cudaEventElapsedTime(&x, pe.second.first, pe.second.second));
            t_ms[pe.first] += x;
            t_n[pe.first] += 1;
            ev_pool.push_back(pe.second.first);
            ev_pool.push_back(pe.second.second);
        }
        ev_pending.clear();
        if (ms) *ms = t_ms[k];
        if (n) *n = t_n[k];
        if (reset)
            for (int j = 0; j < MPS_K_COUNT; ++j) { t_ms[j] = 0; t_n[j] = 0; }
    }

    ~Solver() override {
        for (int b = 0; b < 2; ++b) {
            if (gx_head[b]) cudaGraphExecDestroy(gx_head[b]);
            if (gx_tail[b]) cudaGraphExecDestroy(gx_tail[b]);
        }
        for (auto& pe : ev_pending) {
            cudaEventDestroy(pe.second.first);
            cudaEventDestroy(pe.second.second);
        }
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        if (side) {
            cudaStreamSynchronize(side);
            cudaStreamDestroy(side);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (own_stream) {
            cudaStreamSynchronize(own_stream);
            cudaStreamDestroy(own_stream);
        }
    }

    int dead() const { return C; }
    int L() const { return C + 1; }
    // fluid: fine cells
    int deadF() const { return CF; }
    int LF() const { return CF + 1; }
    int blocks(int n, int b) const { return std::max(1, (n + b - 1) / b); }

    void init(int ns, const mps_params* p, const int32_t* cnts, const int8_t* typ_in,
              const R* pos, const R* vel, const R* nrm) {
        CK(cudaGetDevice(&dev));
        // a stream of its own: the legacy default stream cannot be captured into a graph
        CK(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
        stream = own_stream;
        ensure_side();  // before any capture: stream creation is kept out of graphs
        nscene = ns;
        precision = p[0].precision;
        counts.assign(cnts, cnts + ns);
        nT = 0;
        for (int s = 0; s < ns; ++s) nT += cnts[s];
        hsc.resize(ns);
        infos.resize(ns);
        long long cb = 0, fb = 0;
        int pb = 0;
        for (int s = 0; s < ns; ++s) {
            // each scene's grid fits (derive_scene checks it); the sum over scenes is checked
            // before its base offsets are used
            if (fb + 27LL + 2 > kMaxFineCells)
                throw ApiError(MPS_ERR_OVERFLOW, "the scenes' fine cell grids need more cells "
                                                 "than an int32 index holds");
            derive_scene<R, RN>(p[s], int(cb), int(fb), pb, cnts[s], hsc[s], infos[s]);
            cb += infos[s].nbxyz;
            fb += 27LL * infos[s].nbxyz;
            pb += cnts[s];
            if (fb + 2 > kMaxFineCells)
                throw ApiError(MPS_ERR_OVERFLOW, "the fine cell grid needs " + std::to_string(fb) +
                                                     " cells, more than an int32 index holds");
        }
        C = int(cb);
        CF = int(fb);
        // classify particles: walls inside the padded box are static walls, everything
        // else is a fluid-class particle; RdDat drops what lies outside (kernel.cu:117)
        std::vector<int8_t> ty(typ_in, typ_in + nT);
        fluid_ids.clear();
        wall_ids.clear();
        for (int s = 0, id = 0; s < ns; ++s) {
            R maxc[3];
            for (int d = 0; d < 3; ++d) maxc[d] = R(infos[s].maxc[d]);
            for (int k = 0; k < cnts[s]; ++k, ++id) {
                R x = pos[id], y = pos[nT + id], z = pos[2 * size_t(nT) + id];
                bool in = x < maxc[0] && x > hsc[s].minc[0] && y < maxc[1] && y > hsc[s].minc[1] &&
                          z < maxc[2] && z > hsc[s].minc[2];
                int t = ty[id];
                if (t != kGST && t != kFLD && t != kWLL && t != kOBJ && t != kOBJ2)
                    throw ApiError(MPS_ERR_ARG, "particle " + std::to_string(id) + " has type " +
                                                    std::to_string(t));
                bool wall = (t == kWLL || t == kOBJ || t == kOBJ2);
                if (!in) ty[id] = kGST;
                if (wall && in) wall_ids.push_back(id);
                else fluid_ids.push_back(id);
            }
        }
        nF = int(fluid_ids.size());
        nW = int(wall_ids.size());
        cap = std::max(1024, kNumMRR * nF);
        allocate();
        CK(cudaMemcpyAsync(d_sc, hsc.data(), sizeof(SD) * ns, cudaMemcpyHostToDevice, stream));
        std::vector<int> nb(ns);
        for (int s = 0; s < ns; ++s) nb[s] = infos[s].nbxyz;
        CK(cudaMemcpyAsync(d_nbxyz, nb.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, stream));
        if (nF > 0)
            CK(cudaMemcpyAsync(d_fluid_ids, fluid_ids.data(), sizeof(int) * nF,
                               cudaMemcpyHostToDevice, stream));
        if (nW > 0)
            CK(cudaMemcpyAsync(d_wall_ids, wall_ids.data(), sizeof(int) * nW,
                               cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_nF, &nF, sizeof(int), cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(cnt, 0, sizeof(DevCounters), stream));
        CK(cudaMemsetAsync(diag, 0, sizeof(int32_t) * kDiagCols * size_t(nT), stream));
        CK(cudaMemsetAsync(ndens, 0, sizeof(RN) * size_t(nT), stream));
        // upload: nrm goes through the acc staging buffer
        const size_t n3 = 3 * size_t(nT) * sizeof(R);
        CK(cudaMemcpyAsync(io.pos, pos, n3, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(io.vel, vel, n3, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(io.acc, nrm, n3, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(io.typ, ty.data(), nT, cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(io.prs, 0, sizeof(R) * nT, stream));
        CK(cudaMemsetAsync(io.pav, 0, sizeof(R) * nT, stream));
        if (nW > 0) {
            // walls: unsorted copy in id order, then one bucket build into w_*
            V4<R>* sp = ar.template get<V4<R>>(3 * size_t(nW));
            tw_pos = sp;
            tw_vel = sp + nW;
            tw_nrm = sp + 2 * size_t(nW);
            tw_typ = ar.template get<int8_t>(nW);
            tw_id = ar.template get<int>(nW);
            k_load_walls<R><<<blocks(nW, 256), 256, 0, stream>>>(nT, io.pos, io.vel, io.acc, io.typ,
                                                                 d_wall_ids, nW, tw_pos, tw_vel,
                                                                 tw_nrm, tw_id, tw_typ);
            KL();
            bin_walls();
        } else {
            CK(cudaMemsetAsync(wcs, 0, sizeof(int) * (L() + 1), stream));
            near_wall_flags();
        }
        load_fluid(false);
        mkbkt(true);
        CK(cudaStreamSynchronize(stream));
        Tuned t;
        if (tuned_cache_get(tune_key(), &t)) {
            for (int k = 0; k < MPS_K_COUNT; ++k) blk[k] = t.blk[k];
            stage_mode = t.stage;
            batch_a = t.batch;
            reg_bound = t.regb;
        }
    }

    void allocate() {
        const size_t F = std::max(nF, 1), W = std::max(nW, 1), T = std::max(nT, 1);
        d_sc = ar.template get<SD>(nscene);
        d_nbxyz = ar.template get<int>(nscene);
        for (FluidBuf<R>* b : {&S, &S2}) {
            b->pos = ar.template get<V4<R>>(F);
            b->vel = ar.template get<V4<R>>(F);
            if (b == &S) sbuf0 = b->pos;
            b->acc = ar.template get<V4<R>>(F);
            b->prs = ar.template get<R>(F);
            b->pav = ar.template get<R>(F);
            b->pid = ar.template get<int>(F);
            b->typ = ar.template get<int8_t>(F);
        }
        t_pos = ar.template get<V4<R>>(F);
        t_vel = ar.template get<V4<R>>(F);
        t_prs = ar.template get<R>(F);
        t_typ = ar.template get<int8_t>(F);
        w_pos = ar.template get<V4<R>>(W);
        w_nrm = ar.template get<V4<R>>(W);
        w_vel = ar.template get<V4<R>>(W);
        w_id = ar.template get<int>(W);
        w_typ = ar.template get<int8_t>(W);
        w_se = ar.template get<int8_t>(W);
        wcs = ar.template get<int>(L() + 1);
        cs = ar.template get<int>(size_t(LF()) + 1);
        csr = ar.template get<int>(size_t(LF()) + 1);
        // the fluid's own count table: the start-table pass leaves it zero for the next build
        count_f = ar.template get<int>(size_t(LF()));
        CK(cudaMemsetAsync(count_f, 0, sizeof(int) * size_t(LF()), stream));
        {
            std::vector<int> rs(nscene + 1, 0);
            for (int s = 0; s < nscene; ++s) rs[s + 1] = rs[s] + hsc[s].nby * hsc[s].nbz;
            nrows = rs[nscene];
            int nbx_max = 0;
            for (int s = 0; s < nscene; ++s) nbx_max = std::max(nbx_max, hsc[s].nbx);
            row_threads = nbx_max <= 64 ? 64 : (nbx_max <= 128 ? 128 : 256);
            row_scan = ar.template get<int>(rs.size());
            row_tot = ar.template get<int>(size_t(nrows));
            frow_tot = ar.template get<int>(9 * size_t(nrows));
            CK(cudaMemcpyAsync(row_scan, rs.data(), sizeof(int) * rs.size(), cudaMemcpyHostToDevice,
                               stream));
            CK(cudaStreamSynchronize(stream));  // rs leaves scope
        }
        posf = ar.template get<V4<R>>(F);
        for (MirrorBuf<R>* b : {&U, &M1, &M2}) {
            b->pos = ar.template get<V4<R>>(cap);
            b->slot = ar.template get<int>(cap);
        }
        mcs1 = ar.template get<int>(L() + 1);
        mcs2 = ar.template get<int>(L() + 1);
        const size_t items = std::max<size_t>({F, W, size_t(cap)});
        key = ar.template get<int>(items);
        rnk = ar.template get<int>(items);
        seg = ar.template get<int>(items);
        count = ar.template get<int>(L());
        part = ar.template get<int>((L() + kScan16Tile - 1) / kScan16Tile + 1);
        CK(cudaMemsetAsync(count, 0, sizeof(int) * L(), stream));
        CK(cudaMemsetAsync(part, 0, sizeof(int) * ((L() + kScan16Tile - 1) / kScan16Tile + 1), stream));
        d_fluid_ids = ar.template get<int>(F);
        d_wall_ids = ar.template get<int>(W);
        d_nF = ar.template get<int>(1);
        cnt = ar.template get<DevCounters>(1);
        diag = ar.template get<int32_t>(kDiagCols * T);
        ndens = ar.template get<RN>(T);
        io.n = nT;
        io.pos = ar.template get<R>(3 * T);
        io.vel = ar.template get<R>(3 * T);
        io.acc = ar.template get<R>(3 * T);
        io.prs = ar.template get<R>(T);
        io.pav = ar.template get<R>(T);
        io.typ = ar.template get<int8_t>(T);
        io.cell = ar.template get<int>(T);
        d_integ = ar.template get<double>(6 * size_t(nscene));
        nb = ar.template get<int>(size_t(kListCap) * ((F + 31) / 32 * 32));  // list_at tiles
        near_wall = ar.template get<int8_t>(L());
        near_m1 = ar.template get<int8_t>(L());
        near_m2 = ar.template get<int8_t>(L());
        nbcnt = ar.template get<int>(F);
        CK(cudaMemsetAsync(S.acc, 0, sizeof(V4<R>) * F, stream));
        CK(cudaMemsetAsync(S2.acc, 0, sizeof(V4<R>) * F, stream));
        CK(cudaMemsetAsync(M1.slot, 0, sizeof(int) * cap, stream));
        CK(cudaMemsetAsync(mcs1, 0, sizeof(int) * (L() + 1), stream));
        CK(cudaMemsetAsync(mcs2, 0, sizeof(int) * (L() + 1), stream));
        CK(cudaMemsetAsync(near_m1, 1, L(), stream));  // walk everywhere until a mirror build
        CK(cudaMemsetAsync(near_m2, 1, L(), stream));
    }

    // ---- bucket build ------------------------------------------------------------------
    // bucket build over `ncell` cells (the last one, `ncell - 1`, holds unlisted items)
    template <class Src, class G>
    // (count and part are zero between builds: the scan clears them)
    void bin(Src src, G g, const int* n_ptr, int n_max, int* out_cs, int ncell) {
        if (n_max > 0) {
            int grid = std::min(blocks(n_max, 256), 148 * 32);
            k_bin_key<Src><<<grid, 256, 0, stream>>>(src, n_ptr, n_max, key, rnk, count, part, cnt);
            KL();
        }
        const int nb = (ncell + kScan16Tile - 1) / kScan16Tile;
        FineScan fs{{count, count}, {part, part}, {out_cs, out_cs}, ncell, nb, &cnt->scan_ticket};
        k_fine_scan<<<dim3(nb, 1), kScan16Threads, 0, stream>>>(fs);
        KL();
        if (n_max > 0) {
            int grid = std::min(blocks(n_max, 256), 148 * 32);
            k_bin_seg<Src><<<grid, 256, 0, stream>>>(src, n_ptr, n_max, key, rnk, out_cs, seg);
            KL();
            k_bin_fin<Src, G><<<grid, 256, 0, stream>>>(src, g, n_ptr, n_max, key, rnk, out_cs, seg,
                                                        ncell - 1);
            KL();
        }
    }

    // fluid bucket build from (pos, vel, typ) sources into S2, then S <-> S2
    // The sorted state S2 is bucket-major in fine cells (start table cs); the same build
    // also writes the row-major copy posf (start table csr) that the neighbour walks read.
    void bin_fluid(const V4<R>* pos, const V4<R>* vel, const V4<R>* acc, const R* prs,
                   const R* pav, const int* pid, const int8_t* typ) {
        Scope sc_(this, MPS_K_BIN_FLUID);
        FluidKeySrc<R, RN> ks{d_sc, nscene, deadF(), pos, typ, pid};
        FluidGatherF<R, RN> g{{pos, vel, acc, prs, pav, pid, typ, S2.pos, S2.vel, S2.acc, S2.prs,
                               S2.pav, S2.pid, S2.typ},
                              d_sc, nscene, key, cs, csr, posf};
        const int grid = std::min(blocks(std::max(nF, 1), 256), 148 * 32);
        if (nF > 0) {
            k_bin_key<FluidKeySrc<R, RN>><<<grid, 256, 0, stream>>>(ks, nullptr, nF, key, rnk,
                                                                    count_f, nullptr, cnt);
            KL();
        }
        FineRows fr{count_f, row_tot, frow_tot, cs, csr, row_scan, nscene, nrows, deadF()};
        if (row_threads == 64) fine_rows<64>(fr);
        else if (row_threads == 128) fine_rows<128>(fr);
        else fine_rows<256>(fr);
        if (nF > 0) {
            k_bin_seg<FluidKeySrc<R, RN>><<<grid, 256, 0, stream>>>(ks, nullptr, nF, key, rnk, cs, seg);
            KL();
            k_bin_fin<FluidKeySrc<R, RN>, FluidGatherF<R, RN>><<<grid, 256, 0, stream>>>(
                ks, g, nullptr, nF, key, rnk, cs, seg, deadF());
            KL();
        }
        std::swap(S, S2);
        ++swap_count;
        posf_stale = false;
    }

    template <int T> void fine_rows(const FineRows& fr) {
        k_fine_rows_sum<R, RN, T><<<nrows, T, 0, stream>>>(fr, d_sc);
        KL();
        k_fine_rows_scan<<<2, 1024, 0, stream>>>(fr);
        KL();
        k_fine_rows_write<R, RN, T><<<nrows, T, 0, stream>>>(fr, d_sc);
        KL();
    }

    void mkbkt(bool with_acc) {
        bin_fluid(S.pos, S.vel, with_acc ? S.acc : nullptr, S.prs, S.pav, S.pid, S.typ);
        lists_valid = sorted = true;
    }

    void bin_mirrors(MirrorBuf<R>& dst, int* dcs) {
        Scope sc_(this, MPS_K_BIN_MIRROR);
        MirrorKeySrc<R, RN> ks{d_sc, nscene, dead(), U.pos, U.slot};
        MirrorGather<R> g{U.pos, U.slot, dst.pos, dst.slot};
        bin(ks, g, &cnt->mirror_raw, cap, dcs, L());
        if (dcs == mcs1 || dcs == mcs2) near_flags(dcs, dcs == mcs1 ? near_m1 : near_m2);
    }

    WallView<R> wall_view() const { return WallView<R>{wcs, w_pos, w_nrm, w_vel, w_se, w_typ}; }

    PassArgs<R, RN> args(const MirrorBuf<R>& m, const int* mcs) {
        PassArgs<R, RN> a;
        a.sc = d_sc; a.nscene = nscene; a.nF = nF; a.dead = deadF();
        a.skip = (skip_opt && sorted) ? 1 : 0;
        a.cs = cs;
        a.posf = posf;
        a.csr = csr;
        a.pos = S.pos; a.vel = S.vel; a.acc = S.acc; a.prs = S.prs; a.pav = S.pav; a.pid = S.pid;
        a.typ = S.typ;
        a.tpos = t_pos; a.tvel = t_vel; a.tprs = t_prs; a.ttyp = t_typ;
        a.wl = wall_view();
        a.m = MirrorView<R>{mcs, m.pos, m.slot};
        a.out = MirrorSink<R>{U.pos, U.slot, cap, nullptr};
        a.cnt = cnt; a.diag = diag; a.ndens = ndens;
        a.nb = nb; a.nbcnt = nbcnt; a.nbK = nbK;
        a.near_wall = near_wall;
        a.near_m = mcs == mcs1 ? near_m1 : (mcs == mcs2 ? near_m2 : nullptr);
        a.tape_pre = nullptr;
        return a;
    }

    void reset_raw() { CK(cudaMemsetAsync(&cnt->mirror_raw, 0, sizeof(int), stream)); }

    // MRRinout over the raw mirrors, one thread per mirror (culled slots turn negative)
    void cull_raw() {
        k_ph_cull<R, RN><<<std::min(blocks(4 * cap, 256), 148 * 32), 256, 0, stream>>>(args(M1, mcs1));
        KL();
    }


    // wall bucket build from the load-order copy, then Surface_Edge (kernel.cu:553-668) and
    // the near-wall flags of every bucket
    void bin_walls() {
        WallKeySrc<R, RN> ks{d_sc, nscene, dead(), tw_pos, tw_id};
        WallGather<R> g{tw_pos, tw_nrm, tw_vel, tw_id, tw_typ, w_pos, w_nrm, w_vel, w_id, w_typ};
        bin(ks, g, nullptr, nW, wcs, L());
        k_surface_edge<R, RN><<<blocks(nW, 128), 128, 0, stream>>>(d_sc, nscene, nW, wall_view(),
                                                                   w_id, w_se);
        KL();
        near_wall_flags();
    }

    void near_wall_flags() { near_flags(wcs, near_wall); }
    void near_flags(const int* table_cs, int8_t* out) {
        int nb_max = 1;  // blocks along x cover the largest scene's buckets (y: the scenes)
        for (int s = 0; s < nscene; ++s) nb_max = std::max(nb_max, hsc[s].nbxy * hsc[s].nbz);
        dim3 g(std::max(1, std::min(blocks(nb_max, 256), 148 * 4)), nscene);
        k_near_wall<R, RN><<<g, 256, 0, stream>>>(d_sc, nscene, table_cs, out);
        KL();
    }

    // one step of the moving walls, then their buckets, edge flags and near-wall flags
    void move_walls() {
        k_motion_advance<<<1, 1, 0, stream>>>(d_motion);
        KL();
        k_move_walls<R><<<blocks(nW, 256), 256, 0, stream>>>(d_motion, nW, tw_typ, mx0, mn0, tw_pos,
                                                             tw_nrm, tw_vel);
        KL();
        bin_walls();
    }

    void set_wall_motion(int type, const double* c, const double* axis, double omega,
                         const double* v) override {
        if (type != kOBJ && type != kOBJ2)
            throw ApiError(MPS_ERR_ARG, "only MPS_OBJ and MPS_OBJ2 walls move");
        if (nscene != 1)
            throw ApiError(MPS_ERR_UNSUPPORTED, "wall motion needs a single-scene handle");
        if (!c || !v || (omega != 0.0 && !axis))
            throw ApiError(MPS_ERR_ARG, "centre and velocity (and the axis of a rotation) are needed");
        WallMotion w = wall_motion(type, c, axis, omega, v, double(hsc[0].dt));
        if (!d_motion) {
            d_motion = ar.template get<WallMotion>(2);
            mx0 = ar.template get<double>(3 * size_t(std::max(nW, 1)));
            mn0 = ar.template get<double>(3 * size_t(std::max(nW, 1)));
        }
        const int k = type == kOBJ ? 0 : 1;
        if (w.type != 0 && nW > 0) {
            k_motion_snapshot<R><<<blocks(nW, 256), 256, 0, stream>>>(nW, tw_typ, type, tw_pos,
                                                                      tw_nrm, mx0, mn0);
            KL();
        }
        hmot[k] = w;
        CK(cudaMemcpyAsync(d_motion, hmot, sizeof(hmot), cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));
        motion_on = nW > 0 && (hmot[0].type != 0 || hmot[1].type != 0);
        invalidate_graph();
    }

    // capacity of a block's stage: the option, else what keeps four blocks per SM
    int staged_capacity() const {
        if (stage_cap > 0) return stage_cap;
        const bool v = stage_mode == MPS_STAGE_VELOCITIES;
        const size_t budget = 227 * 1024 / 4 - ((sizeof(StageHdr) + 15) / 16) * 16 - 1024;
        return int(budget / (sizeof(V4<R>) * (v ? 2 : 1)));
    }
    template <bool D, bool SV> void launch_pass_a_staged_v(int ba) {
        const int cap = staged_capacity();
        const size_t bytes = stage_smem_bytes<R>(cap, SV);
        CK(cudaFuncSetAttribute(k_pass_a_st<R, RN, D, SV>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
        k_pass_a_st<R, RN, D, SV><<<blocks(nF, ba), ba, bytes, stream>>>(args(M1, mcs1), cap);
    }
    template <bool D> void launch_pass_a_staged(int ba) {
        if (stage_mode == MPS_STAGE_VELOCITIES) launch_pass_a_staged_v<D, true>(ba);
        else launch_pass_a_staged_v<D, false>(ba);
    }

    // pass A walking global memory, at the handle's candidate batch
    template <bool D, bool ALT> void launch_pass_a(int ba) {
        if (batch_a == 2)
            k_pass_a<R, RN, D, false, 2, ALT><<<blocks(nF, ba), ba, 0, stream>>>(args(M1, mcs1));
        else if (batch_a == 8)
            k_pass_a<R, RN, D, false, 8, ALT><<<blocks(nF, ba), ba, 0, stream>>>(args(M1, mcs1));
        else
            k_pass_a<R, RN, D, false, 4, ALT><<<blocks(nF, ba), ba, 0, stream>>>(args(M1, mcs1));
    }

    template <bool D> void fused_body() {
        const int ba = blk[MPS_K_PASS_A], bb = blk[MPS_K_PASS_B], bc = blk[MPS_K_PASS_C],
                  bg = blk[MPS_K_GEN];
        // pass A: VscTrm + UpPcl1
        {
            Scope t(this, MPS_K_PASS_A);
            if (stage_mode != MPS_STAGE_GLOBAL)
                launch_pass_a_staged<D>(ba);
            else if (reg_bound & 4)
                launch_pass_a<D, true>(ba);
            else
                launch_pass_a<D, false>(ba);
            KL();
        }
        // MkBkt on x* (kernel.cu:1917); the rebuild at kernel.cu:1921 would give the same lists
        bin_fluid(t_pos, t_vel, nullptr, S.prs, S.pav, S.pid, t_typ);
        // The step's second mirror generation (the one the reference's counters would show
        // last) is made at (x*, P): its positions, cull and bucket build need only x*, which
        // ChkCol does not move (it changes velocities only, kernel.cu:1281-1287), and read
        // nothing pass B writes; pass B reads the first generation's table M1, not the raw
        // list, M2 or their scratch. So with bit 1 of overlap they run on the second stream
        // beside pass B, and k_mirror_prs fills in the pressures once pass B has made them.
        const bool fork = (overlap & 2) && !timing_on;
        if (fork) {
            CK(cudaEventRecord(ev_fork, stream));
            CK(cudaStreamWaitEvent(side, ev_fork, 0));
            OnStream o(this, side);
            reset_raw();
            {
                Scope t(this, MPS_K_GEN);
                k_gen_cull<R, RN, D><<<blocks(nF, bg), bg, 0, stream>>>(args(M1, mcs1), S.pos,
                                                                               nullptr, S.typ);
                KL();
                cull_raw();
            }
            bin_mirrors(M2, mcs2);
            CK(cudaEventRecord(ev_join, side));
        }
        // pass B: ChkCol + MkPrs
        {
            Scope t(this, MPS_K_PASS_B);
            if (reg_bound & 1)
                k_pass_b<R, RN, D, true><<<blocks(nF, bb), bb, 0, stream>>>(args(M1, mcs1));
            else
                k_pass_b<R, RN, D><<<blocks(nF, bb), bb, 0, stream>>>(args(M1, mcs1));
            KL();
        }
        if (fork) {
            CK(cudaStreamWaitEvent(stream, ev_join, 0));
            k_mirror_prs<R><<<std::min(blocks(std::max(cap, 1), 256), 148 * 8), 256, 0, stream>>>(
                mcs2, dead(), M2.pos, t_prs, nF);
            KL();
        } else {
            reset_raw();
            {
                Scope t(this, MPS_K_GEN);
                k_gen_cull<R, RN, D><<<blocks(nF, bg), bg, 0, stream>>>(args(M1, mcs1), S.pos,
                                                                               t_prs, S.typ);
                KL();
                cull_raw();
            }
            bin_mirrors(M2, mcs2);
        }
        // pass C: PrsGrdTrm + UpPcl2, then the first mirror generation of the next step
        {
            Scope t(this, MPS_K_PASS_C);
            if (grad_mode == MPS_GRAD_CORRECTED)
                k_pass_c<R, RN, D, false, true><<<blocks(nF, bc), bc, 0, stream>>>(args(M2, mcs2));
            else if (reg_bound & 2)
                k_pass_c<R, RN, D, false, false, true><<<blocks(nF, bc), bc, 0, stream>>>(
                    args(M2, mcs2));
            else
                k_pass_c<R, RN, D><<<blocks(nF, bc), bc, 0, stream>>>(args(M2, mcs2));
            KL();
        }
        // walls that move take their place at the new time before the next step's mirrors
        if (motion_on) move_walls();
    }

    // the end of a step: the next step's first mirror generation at x^{n+1}, then the bucket
    // builds of x^{n+1} and of those mirrors
    // The generation reads t_pos, t_prs, t_typ, the pre-build S.pid, the walls and the near
    // flags and writes the raw mirrors; the fluid build reads the same t_* and S arrays and
    // writes S2, its start tables, posf and its own key/rank scratch. Neither writes what the
    // other reads, so with overlap_on the build runs on the second stream beside the
    // generation and its cull, and the mirror bucket build (which reuses the key/rank
    // scratch) waits for both. Both launches are issued before the build swaps S and S2 on
    // the host, so the generation's arguments name the pre-build arrays either way.
    void step_tail() {
        const int bg = blk[MPS_K_GEN];
        const bool fork = (overlap & 1) && !timing_on;
        reset_raw();
        if (fork) {
            ensure_side();
            CK(cudaEventRecord(ev_fork, stream));
            CK(cudaStreamWaitEvent(side, ev_fork, 0));
        }
        {
            Scope t(this, MPS_K_GEN);
            k_gen_cull<R, RN, false><<<blocks(nF, bg), bg, 0, stream>>>(args(M2, mcs2), t_pos,
                                                                               t_prs, t_typ);
            KL();
            cull_raw();
        }
        if (fork) {
            {
                OnStream o(this, side);
                bin_fluid(t_pos, t_vel, nullptr, t_prs, S.pav, S.pid, t_typ);
                CK(cudaEventRecord(ev_join, side));
            }
            CK(cudaStreamWaitEvent(stream, ev_join, 0));
        } else {
            bin_fluid(t_pos, t_vel, nullptr, t_prs, S.pav, S.pid, t_typ);
        }
        bin_mirrors(M1, mcs1);
    }

    // runs the pending end of the latest step, if any (before reading the sorted state)
    void finish_tail() {
        if (!tail_pending) return;
        step_tail();
        tail_pending = false;
    }

    void prepare_fused() {
        if (!lists_valid || !sorted) mkbkt(acc_dirty);
        if (acc_dirty) {
            CK(cudaMemsetAsync(S.acc, 0, sizeof(V4<R>) * std::max(nF, 1), stream));
            CK(cudaMemsetAsync(S2.acc, 0, sizeof(V4<R>) * std::max(nF, 1), stream));
            acc_dirty = false;
        }
        if (!m1_valid) {
            reset_raw();
            k_gen_cull<R, RN, false><<<blocks(nF, block), block, 0, stream>>>(
                args(M1, mcs1), S.pos, S.prs, S.typ);
            KL();
            cull_raw();
            bin_mirrors(M1, mcs1);
            m1_valid = true;
        }
    }

    // one instantiated CUDA graph of `body`'s launches; `nl` receives their count
    template <class F> void capture(cudaGraphExec_t& ge, long long& nl, int& nswap, F&& body) {
        cudaGraph_t g;
        const long long l0 = launches;
        const int s0 = swap_count;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            body();
        } catch (...) {
            cudaStreamEndCapture(stream, &g);
            throw;
        }
        CK(cudaStreamEndCapture(stream, &g));
        nl = launches - l0;
        nswap = swap_count - s0;
        launches = l0;  // captured, not yet run
        cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        CK(e);
    }

    void run_body() {
        if (diag_on) fused_body<true>(); else fused_body<false>();
    }

    // Autotuner. Candidates per kernel group, each timed over `trial` steps with CUDA events:
    //   pass A (VscTrm): candidates in flight (2, 4, 8) and 128 or 64 threads per block
    //                    for the walk through L1, and the staged walk at 128 threads;
    //   passes B, C and mirror generation: 128, 96, 64 or 32 threads per block;
    //   then passes B, C and A at their alternate register bound, with the chosen shapes
    //   (pass A with each candidate batch).
    // All groups are timed in the same trial steps (they are separate kernels), and every
    // round starts from the handle's state (restored from a snapshot). The state is
    // restored afterwards, and the choice is kept for later handles of the same precision
    // and size class in this process (tuned_cache).
    void autotune(int trial, int32_t* chosen) override {
        finish_tail();
        struct CandA { int blk, stage, batch; };
        const CandA cand_a[] = {{128, MPS_STAGE_GLOBAL, 4}, {64, MPS_STAGE_GLOBAL, 4},
                                {128, MPS_STAGE_GLOBAL, 2}, {64, MPS_STAGE_GLOBAL, 2},
                                {128, MPS_STAGE_GLOBAL, 8}, {128, MPS_STAGE_POSITIONS, 4}};
        const int cand_b[] = {128, 96, 64, 32};
        const int groups_b[] = {MPS_K_PASS_B, MPS_K_PASS_C, MPS_K_GEN};
        double best[MPS_K_COUNT];
        int bestb[MPS_K_COUNT];
        for (int k = 0; k < MPS_K_COUNT; ++k) { best[k] = 1e300; bestb[k] = blk[k]; }
        int best_stage = stage_mode, best_batch = batch_a;
        reg_bound = 0;
        store_all();  // snapshot of the state in the id-order staging buffers
        const long long steps0 = steps;
        const bool timing0 = timing_on;
        timing_on = true;
        invalidate_graph();
        timing(0, nullptr, nullptr, true);
        const int nround = int(sizeof(cand_a) / sizeof(cand_a[0]));
        for (int i = 0; i < nround; ++i) {
            blk[MPS_K_PASS_A] = cand_a[i].blk;
            stage_mode = cand_a[i].stage;
            batch_a = cand_a[i].batch;
            const bool new_b = i < 4;
            if (new_b)
                for (int g : groups_b) blk[g] = cand_b[i];
            // every candidate runs the same steps from the snapshot (a dam break's steps
            // grow slower as it evolves, which would favour the candidates tried first)
            load_fluid(true);
            step(trial);
            auto read = [&](int g, double& ms_per) {
                double ms = 0;
                long long n = 0;
                timing(g, &ms, &n, false);
                ms_per = n > 0 ? ms / n : 1e300;
            };
            double ms;
            read(MPS_K_PASS_A, ms);
            if (ms < best[MPS_K_PASS_A]) {
                best[MPS_K_PASS_A] = ms;
                bestb[MPS_K_PASS_A] = cand_a[i].blk;
                best_stage = cand_a[i].stage;
                best_batch = cand_a[i].batch;
            }
            if (new_b)
                for (int g : groups_b) {
                    read(g, ms);
                    if (ms < best[g]) { best[g] = ms; bestb[g] = cand_b[i]; }
                }
            timing(0, nullptr, nullptr, true);
        }
        for (int g : groups_b) blk[g] = bestb[g];
        blk[MPS_K_PASS_A] = bestb[MPS_K_PASS_A];
        stage_mode = best_stage;
        batch_a = best_batch;
        // the alternate register bounds of passes B, C and A, at the chosen shapes; pass A's
        // bound and its candidate batch interact (fewer registers suit a smaller batch), so
        // pass A tries the alternate bound with every batch
        int regb = 0;
        const int chosen_batch = batch_a;
        const int batches[3] = {chosen_batch, chosen_batch == 2 ? 4 : 2, chosen_batch == 8 ? 4 : 8};
        for (int r = 0; r < 3; ++r) {
            reg_bound = 7;
            batch_a = batches[r];
            load_fluid(true);
            step(trial);
            double ms = 0;
            long long n = 0;
            if (r == 0) {
                timing(MPS_K_PASS_B, &ms, &n, false);
                if (n > 0 && ms / n < best[MPS_K_PASS_B]) regb |= 1;
                ms = 0;
                n = 0;
                timing(MPS_K_PASS_C, &ms, &n, false);
                if (n > 0 && ms / n < best[MPS_K_PASS_C]) regb |= 2;
                ms = 0;
                n = 0;
            }
            timing(MPS_K_PASS_A, &ms, &n, false);
            if (stage_mode == MPS_STAGE_GLOBAL && n > 0 && ms / n < best[MPS_K_PASS_A]) {
                best[MPS_K_PASS_A] = ms / n;
                regb |= 4;
                best_batch = batches[r];
            }
            timing(0, nullptr, nullptr, true);
        }
        batch_a = best_batch;
        reg_bound = regb;
        load_fluid(true);  // back to the snapshot: tuning leaves no trace in the results
        steps = steps0;
        timing_on = timing0;
        invalidate_graph();
        CK(cudaStreamSynchronize(stream));
        tuned_cache_put(tune_key(), Tuned{{blk[0], blk[1], blk[2], blk[3], blk[4], blk[5]},
                                          stage_mode, batch_a, reg_bound});
        if (chosen)
            for (int k = 0; k < MPS_K_COUNT; ++k) chosen[k] = blk[k];
    }

    // size class of the handle for the tuning cache: precision, batched or not, log2 of the
    // fluid count
    TuneKey tune_key() const {
        int lg = 0;
        while ((2LL << lg) <= (long long)std::max(nF, 1)) ++lg;
        return TuneKey{precision, nscene > 1 ? 1 : 0, lg};
    }

    int list_capacity() const override { return nbK; }

    void set_list_capacity(int k) override {
        nbK = (k == 0 || k > kListCap) ? kListCap : k;
        invalidate_graph();  // the captured launches carry the capacity
    }

    void invalidate_graph() override {
        for (int b = 0; b < 2; ++b) {
            if (gx_head[b]) cudaGraphExecDestroy(gx_head[b]);
            if (gx_tail[b]) cudaGraphExecDestroy(gx_tail[b]);
            gx_head[b] = gx_tail[b] = nullptr;
        }
    }

    // Launches the graph of `body` for the buffer the sorted state is in, capturing it first
    // if needed (the capture runs the host side of `body`, its swaps included); a replay
    // repeats the captured swaps on the host.
    template <class F>
    void run_graph(cudaGraphExec_t* gx, long long& nl, int& nswap, F&& body) {
        const int b = S.pos == sbuf0 ? 0 : 1;
        if (!gx[b]) {
            capture(gx[b], nl, nswap, body);
        } else {
            for (int k = 0; k < nswap; ++k) std::swap(S, S2);
            swap_count += nswap;
            if (nswap) posf_stale = false;
        }
        CK(cudaGraphLaunch(gx[b], stream));
        launches += nl;
    }

    // A step is its body (passes A to C) preceded by the end of the step before it, or by a
    // full bucket build and mirror generation when the state was set or changed since.
    void step(int n) override {
        if (n <= 0) return;
        const bool use_graph = graph_on && !timing_on;
        if (gexec_diag != diag_on) invalidate_graph();
        gexec_diag = diag_on;
        for (int k = 0; k < n; ++k) {
            if (tail_pending) {
                if (use_graph) run_graph(gx_tail, tail_launches, swaps_tail, [&] { step_tail(); });
                else step_tail();
                tail_pending = false;
            } else if (!(lists_valid && sorted && m1_valid) || acc_dirty) {
                prepare_fused();
            }
            if (use_graph) run_graph(gx_head, head_launches, swaps_head, [&] { run_body(); });
            else run_body();
            tail_pending = true;
            lists_valid = sorted = m1_valid = true;  // as the pending end will leave them
        }
        steps += n;
    }

    void phase(int ph) override {
        finish_tail();
        PassArgs<R, RN> a = args(M1, mcs1);
        const int gb = blocks(nF, block);
        auto need_lists = [&]() {
            if (!lists_valid)
                throw ApiError(MPS_ERR_STATE, "bucket lists are not built: run MPS_PHASE_MKBKT first");
            if (posf_stale) {  // the lists stay, the positions read through them are current
                k_posf_refresh<R><<<std::min(blocks(std::max(nF, 1), 256), 148 * 8), 256, 0, stream>>>(
                    posf, S.pos, csr, deadF());
                KL();
                posf_stale = false;
            }
        };
        m1_valid = false;
        switch (ph) {
            case MPS_PHASE_MKBKT:
                mkbkt(true);
                break;
            case MPS_PHASE_SURFACE_EDGE:
                if (nW > 0) {
                    k_surface_edge<R, RN><<<blocks(nW, 128), 128, 0, stream>>>(d_sc, nscene, nW,
                                                                               wall_view(), w_id, w_se);
                    KL();
                }
                break;
            case MPS_PHASE_RESETMRR:
                reset_raw();
                break;
            case MPS_PHASE_GENMRR_NONSLIP:
                if (diag_on) k_ph_gen<R, RN, true><<<gb, block, 0, stream>>>(a);
                else k_ph_gen<R, RN, false><<<gb, block, 0, stream>>>(a);
                KL();
                break;
            case MPS_PHASE_MKBKT_MRR:
                cull_raw();
                bin_mirrors(M1, mcs1);
                break;
            case MPS_PHASE_VSCTRM:
                need_lists();
                if (diag_on) k_ph_vsc<R, RN, true><<<gb, block, 0, stream>>>(a);
                else k_ph_vsc<R, RN, false><<<gb, block, 0, stream>>>(a);
                KL();
                acc_dirty = true;
                break;
            case MPS_PHASE_UPPCL1:
                k_ph_uppcl1<R, RN><<<gb, block, 0, stream>>>(a);
                KL();
                sorted = false;
                posf_stale = true;
                acc_dirty = true;
                break;
            case MPS_PHASE_CHKCOL:
                need_lists();
                if (diag_on) k_ph_col<R, RN, true><<<gb, block, 0, stream>>>(a);
                else k_ph_col<R, RN, false><<<gb, block, 0, stream>>>(a);
                KL();
                k_ph_upchkcol<R, RN><<<gb, block, 0, stream>>>(a);
                KL();
                acc_dirty = true;
                break;
            case MPS_PHASE_MKPRS:
                need_lists();
                if (diag_on) k_ph_prs<R, RN, true><<<gb, block, 0, stream>>>(a);
                else k_ph_prs<R, RN, false><<<gb, block, 0, stream>>>(a);
                KL();
                break;
            case MPS_PHASE_PRSGRDTRM:
                need_lists();
                if (grad_mode == MPS_GRAD_CORRECTED) {
                    if (diag_on) k_ph_grd<R, RN, true, true><<<gb, block, 0, stream>>>(a);
                    else k_ph_grd<R, RN, false, true><<<gb, block, 0, stream>>>(a);
                } else {
                    if (diag_on) k_ph_grd<R, RN, true><<<gb, block, 0, stream>>>(a);
                    else k_ph_grd<R, RN, false><<<gb, block, 0, stream>>>(a);
                }
                KL();
                acc_dirty = true;
                break;
            case MPS_PHASE_UPPCL2:
                k_ph_uppcl2<R, RN><<<gb, block, 0, stream>>>(a);
                KL();
                sorted = false;
                posf_stale = true;
                acc_dirty = true;
                break;
            default:
                throw ApiError(MPS_ERR_ARG, "unknown phase " + std::to_string(ph));
        }
    }

    // ---- state I/O ---------------------------------------------------------------------
    void load_fluid(bool use_acc) {
        k_load_fluid<R><<<blocks(nF, 256), 256, 0, stream>>>(io, d_fluid_ids, nF, S.pos, S.vel,
                                                             S.acc, S.prs, S.pav, S.pid, S.typ,
                                                             use_acc ? 1 : 0);
        KL();
        lists_valid = sorted = m1_valid = false;
        acc_dirty = use_acc;
        tail_pending = false;  // the loaded state replaces what the latest step left
    }

    // the state in id order into io; with a step's end pending, from the arrays pass C left
    // (in S's slot order; acc is zero between steps in both). `mask` (kIo* bits) selects the
    // arrays; the bucket index of each particle (io.cell) comes with kIoCell.
    static constexpr int kIoPos = 1, kIoVel = 2, kIoAcc = 4, kIoPrs = 8, kIoPav = 16,
                         kIoTyp = 32, kIoCell = 64, kIoAll = 127;
    void store_all(int mask = kIoAll) {
        IdState<R> st = io;
        if (!(mask & kIoPos)) st.pos = nullptr;
        if (!(mask & kIoVel)) st.vel = nullptr;
        if (!(mask & kIoAcc)) st.acc = nullptr;
        if (!(mask & kIoPrs)) st.prs = nullptr;
        if (!(mask & kIoPav)) st.pav = nullptr;
        if (!(mask & kIoTyp)) st.typ = nullptr;
        if (!(mask & kIoCell)) st.cell = nullptr;
        if (!(mask & kIoAll)) return;
        if (tail_pending)
            k_store_fluid<R, RN><<<blocks(nF, 256), 256, 0, stream>>>(st, d_sc, nscene, nF, t_pos,
                                                                      t_vel, S.acc, t_prs, S.pav,
                                                                      S.pid, t_typ);
        else
            k_store_fluid<R, RN><<<blocks(nF, 256), 256, 0, stream>>>(st, d_sc, nscene, nF, S.pos,
                                                                      S.vel, S.acc, S.prs, S.pav,
                                                                      S.pid, S.typ);
        KL();
        if (nW > 0) {
            k_store_walls<R, RN><<<blocks(nW, 256), 256, 0, stream>>>(st, d_sc, nscene, nW, w_pos,
                                                                      w_vel, w_id, w_typ);
            KL();
        }
    }

    void get_state(int8_t* typ, void* pos, void* vel, void* acc, void* prs, void* pav) override {
        store_all((typ ? kIoTyp : 0) | (pos ? kIoPos : 0) | (vel ? kIoVel : 0) |
                  (acc ? kIoAcc : 0) | (prs ? kIoPrs : 0) | (pav ? kIoPav : 0));
        const size_t n3 = 3 * size_t(nT) * sizeof(R), n1 = size_t(nT) * sizeof(R);
        if (typ) CK(cudaMemcpyAsync(typ, io.typ, nT, cudaMemcpyDeviceToHost, stream));
        if (pos) CK(cudaMemcpyAsync(pos, io.pos, n3, cudaMemcpyDeviceToHost, stream));
        if (vel) CK(cudaMemcpyAsync(vel, io.vel, n3, cudaMemcpyDeviceToHost, stream));
        if (acc) CK(cudaMemcpyAsync(acc, io.acc, n3, cudaMemcpyDeviceToHost, stream));
        if (prs) CK(cudaMemcpyAsync(prs, io.prs, n1, cudaMemcpyDeviceToHost, stream));
        if (pav) CK(cudaMemcpyAsync(pav, io.pav, n1, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    void set_state(const int8_t* typ, const void* pos, const void* vel, const void* acc,
                   const void* prs, const void* pav) override {
        // start from the current state so that omitted arrays keep their values
        store_all((typ ? 0 : kIoTyp) | (pos ? 0 : kIoPos) | (vel ? 0 : kIoVel) |
                  (acc ? 0 : kIoAcc) | (prs ? 0 : kIoPrs) | (pav ? 0 : kIoPav));
        const size_t n3 = 3 * size_t(nT) * sizeof(R), n1 = size_t(nT) * sizeof(R);
        if (typ) CK(cudaMemcpyAsync(io.typ, typ, nT, cudaMemcpyHostToDevice, stream));
        if (pos) CK(cudaMemcpyAsync(io.pos, pos, n3, cudaMemcpyHostToDevice, stream));
        if (vel) CK(cudaMemcpyAsync(io.vel, vel, n3, cudaMemcpyHostToDevice, stream));
        if (acc) CK(cudaMemcpyAsync(io.acc, acc, n3, cudaMemcpyHostToDevice, stream));
        if (prs) CK(cudaMemcpyAsync(io.prs, prs, n1, cudaMemcpyHostToDevice, stream));
        if (pav) CK(cudaMemcpyAsync(io.pav, pav, n1, cudaMemcpyHostToDevice, stream));
        load_fluid(true);
        CK(cudaStreamSynchronize(stream));
    }

    void output_snapshot(void* pos, void* vel, void* prs, void* pav, int8_t* typ, void* mpos,
                         int* mslot, int* mcount_host) override {
        store_all();
        const size_t n3 = 3 * size_t(nT) * sizeof(R), n1 = size_t(nT) * sizeof(R);
        CK(cudaMemcpyAsync(pos, io.pos, n3, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(vel, io.vel, n3, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(prs, io.prs, n1, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(pav, io.pav, n1, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(typ, io.typ, nT, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(mpos, M2.pos, sizeof(V4<R>) * size_t(cap), cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(mslot, M2.slot, sizeof(int) * size_t(cap), cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(mcount_host, mcs2 + dead(), sizeof(int), cudaMemcpyDeviceToHost, stream));
        // d_initialize_real_array(d_pav, 0) after WrtDat (kernel.cu:289)
        CK(cudaMemsetAsync(S.pav, 0, sizeof(R) * size_t(std::max(nF, 1)), stream));
    }

    void get_wall_normals(void* nrm) override {
        R* o = static_cast<R*>(nrm);
        std::memset(o, 0, 3 * size_t(nT) * sizeof(R));
        if (nW == 0) return;
        std::vector<V4<R>> n(nW);
        std::vector<int> ids(nW);
        CK(cudaMemcpyAsync(n.data(), w_nrm, sizeof(V4<R>) * nW, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(ids.data(), w_id, sizeof(int) * nW, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (int w = 0; w < nW; ++w) {
            o[ids[w]] = n[w].x;
            o[size_t(nT) + ids[w]] = n[w].y;
            o[2 * size_t(nT) + ids[w]] = n[w].z;
        }
    }

    void get_wall_flags(int8_t* out) override {
        std::vector<int8_t> se(std::max(nW, 1));
        if (nW > 0) {
            CK(cudaMemcpyAsync(se.data(), w_se, nW, cudaMemcpyDeviceToHost, stream));
            std::vector<int> ids(nW);
            CK(cudaMemcpyAsync(ids.data(), w_id, sizeof(int) * nW, cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            std::memset(out, 0, nT);
            for (int w = 0; w < nW; ++w) out[ids[w]] = se[w];
        } else {
            std::memset(out, 0, nT);
        }
    }

    int get_mirrors(int which, int cp, int32_t* slot, void* pos, void* prs) override {
        if (which != 2) finish_tail();  // the raw list and M1 are the step end's generation
        int n = 0;
        const MirrorBuf<R>* b = which == 2 ? &M2 : (which == 1 ? &M1 : &U);
        if (which == 0) {
            CK(cudaMemcpyAsync(&n, &cnt->mirror_raw, sizeof(int), cudaMemcpyDeviceToHost, stream));
        } else {
            CK(cudaMemcpyAsync(&n, (which == 2 ? mcs2 : mcs1) + dead(), sizeof(int),
                               cudaMemcpyDeviceToHost, stream));
        }
        CK(cudaStreamSynchronize(stream));
        n = std::min(n, cap);
        std::vector<V4<R>> p(std::max(n, 1));
        std::vector<int> s(std::max(n, 1));
        if (n > 0) {
            CK(cudaMemcpyAsync(p.data(), b->pos, sizeof(V4<R>) * n, cudaMemcpyDeviceToHost, stream));
            CK(cudaMemcpyAsync(s.data(), b->slot, sizeof(int) * n, cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
        }
        std::vector<int> order;
        for (int k = 0; k < n; ++k)
            if (s[k] >= 0) order.push_back(k);
        std::sort(order.begin(), order.end(), [&](int a, int b2) { return s[a] < s[b2]; });
        int m = int(order.size());
        for (int k = 0; k < m && k < cp; ++k) {
            int q = order[k];
            if (slot) slot[k] = s[q];
            if (pos) {
                R* o = static_cast<R*>(pos);
                o[k] = p[q].x; o[cp + k] = p[q].y; o[2 * size_t(cp) + k] = p[q].z;
            }
            if (prs) static_cast<R*>(prs)[k] = p[q].w;
        }
        return m;
    }

    void get_diag(int32_t* table, void* nd) override {
        store_all();  // refreshes io.cell from the current positions
        std::vector<int> cell(nT);
        CK(cudaMemcpyAsync(cell.data(), io.cell, sizeof(int) * nT, cudaMemcpyDeviceToHost, stream));
        if (table)
            CK(cudaMemcpyAsync(table, diag, sizeof(int32_t) * kDiagCols * size_t(nT),
                               cudaMemcpyDeviceToHost, stream));
        std::vector<RN> ndn(nT);
        CK(cudaMemcpyAsync(ndn.data(), ndens, sizeof(RN) * nT, cudaMemcpyDeviceToHost, stream));
        std::vector<int8_t> ty(nT);
        CK(cudaMemcpyAsync(ty.data(), io.typ, nT, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        if (table)
            for (int i = 0; i < nT; ++i) table[size_t(i) * kDiagCols] = ty[i] == kGST ? -1 : cell[i];
        if (nd)
            for (int i = 0; i < nT; ++i) static_cast<R*>(nd)[i] = R(ndn[i]);
    }

    void get_counters(mps_counters* o) override {
        DevCounters c;
        int a1 = 0, a2 = 0, alive = 0;
        CK(cudaMemcpyAsync(&c, cnt, sizeof(c), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(&a1, mcs1 + dead(), sizeof(int), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(&a2, mcs2 + dead(), sizeof(int), cudaMemcpyDeviceToHost, stream));
        std::vector<int8_t> ty(std::max(nF, 1));
        CK(cudaMemcpyAsync(ty.data(), tail_pending ? t_typ : S.typ, std::max(nF, 1),
                           cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (int k = 0; k < nF; ++k) alive += ty[k] == kFLD;
        std::memset(o, 0, sizeof(*o));
        o->steps = steps;
        o->n_fluid_alive = alive;
        o->n_deleted = nF - alive;
        o->n_mirror_1 = a1;
        o->n_mirror_2 = a2;
        o->err_mirror_slot = c.err_mirror_slot;
        o->err_mirror_capacity = c.err_capacity;
        o->err_cell_range = c.err_cell;
        o->err_nan = c.err_nan;
        o->kernel_launches = launches;
        o->stage_blocks = c.stage_blocks;
        o->unstaged_blocks = c.unstaged_blocks;
    }

    void get_work(mps_work* o) override {
        DevCounters c;
        CK(cudaMemcpyAsync(&c, cnt, sizeof(c), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        std::memset(o, 0, sizeof(*o));
        o->visc_candidates = (long long)c.work[0];
        o->list_candidates = (long long)c.work[1];
        o->list_entries = (long long)c.work[2];
    }

    // ---- adjoint of a recorded rollout -------------------------------------------------
    // A rollout of n steps keeps the state every k steps (particle-id order, as the staging
    // buffers hold it). The backward sweep walks the segments last to first: it restores a
    // segment's first state, replays the segment's steps with the recording kernels (which
    // keep the neighbour lists, mirror generations and pre-clamp velocities of each step)
    // and runs the step adjoints in reverse over what they kept. The replay repeats the
    // original steps exactly: the bucket order and every sum depend on the state only.
    struct Ckpt {
        R* pos; R* vel; R* prs; R* pav; int8_t* typ;
    };
    struct AdjState {
        DevArena ar;
        int nsteps = 0, every = 0, nck = 0;
        int nbK = 0;  // list capacity the tape was allocated and recorded with
        long long steps_end = 0;
        std::vector<Ckpt> ck;  // nck segment starts + the final state
        std::vector<TapeStep<R>> tape;
        V4<R>* unrm = nullptr;
        V4<double> *lx, *lv, *lx_acc, *lG, *lvv, *lxs, *lx_at, *lxs_pid, *lu_pid, *la, *lxa, *lva;
        double *lP, *lP_at, *lkn, *stage;
        R* pmin;
        int *am, *inv2, *err;
    };
    std::unique_ptr<AdjState> adj;

    void snapshot(const Ckpt& c) {
        store_all();
        const size_t n3 = 3 * size_t(nT) * sizeof(R), n1 = size_t(nT) * sizeof(R);
        CK(cudaMemcpyAsync(c.pos, io.pos, n3, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(c.vel, io.vel, n3, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(c.prs, io.prs, n1, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(c.pav, io.pav, n1, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(c.typ, io.typ, nT, cudaMemcpyDeviceToDevice, stream));
    }

    void restore(const Ckpt& c) {
        const size_t n3 = 3 * size_t(nT) * sizeof(R), n1 = size_t(nT) * sizeof(R);
        CK(cudaMemcpyAsync(io.pos, c.pos, n3, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(io.vel, c.vel, n3, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(io.prs, c.prs, n1, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(io.pav, c.pav, n1, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(io.typ, c.typ, nT, cudaMemcpyDeviceToDevice, stream));
        load_fluid(false);
    }

    void adj_alloc(int nck, int every) {
        adj.reset();
        auto st = std::make_unique<AdjState>();
        st->nbK = nbK;
        DevArena& a = st->ar;
        const size_t F = std::max(nF, 1), T = std::max(nT, 1), Cm = size_t(cap), Lc = L() + 1;
        const size_t F32 = (F + 31) / 32 * 32;  // slots rounded to whole warps (list_at)
        for (int c = 0; c <= nck; ++c)
            st->ck.push_back(Ckpt{a.template get<R>(3 * T), a.template get<R>(3 * T),
                                  a.template get<R>(T), a.template get<R>(T),
                                  a.template get<int8_t>(T)});
        for (int k = 0; k < every; ++k) {
            TapeStep<R> t;
            t.pid1 = a.template get<int>(F); t.x1 = a.template get<V4<R>>(F);
            t.v1 = a.template get<V4<R>>(F); t.up1 = a.template get<V4<R>>(F);
            t.nA = a.template get<int>(F); t.nbA = a.template get<int>(size_t(nbK) * F32);
            t.m1pos = a.template get<V4<R>>(Cm); t.m1slot = a.template get<int>(Cm);
            t.m1nrm = a.template get<V4<R>>(Cm); t.mcs1 = a.template get<int>(Lc);
            t.pid2 = a.template get<int>(F); t.x2 = a.template get<V4<R>>(F);
            t.u2 = a.template get<V4<R>>(F); t.vv2 = a.template get<V4<R>>(F);
            t.P2 = a.template get<R>(F); t.vp2 = a.template get<V4<R>>(F);
            t.nB = a.template get<int>(F); t.nbB = a.template get<int>(size_t(nbK) * F32);
            t.m2pos = a.template get<V4<R>>(Cm); t.m2slot = a.template get<int>(Cm);
            t.m2nrm = a.template get<V4<R>>(Cm); t.mcs2 = a.template get<int>(Lc);
            st->tape.push_back(t);
        }
        st->unrm = a.template get<V4<R>>(Cm);
        for (V4<double>** p : {&st->lx, &st->lv, &st->lx_acc, &st->lxs_pid, &st->lu_pid})
            *p = a.template get<V4<double>>(T);
        for (V4<double>** p : {&st->lG, &st->lvv, &st->lxs, &st->lx_at, &st->la, &st->lxa, &st->lva})
            *p = a.template get<V4<double>>(F);
        st->lP = a.template get<double>(F);
        st->lP_at = a.template get<double>(F);
        st->lkn = a.template get<double>(1);
        st->stage = a.template get<double>(3 * T);
        st->pmin = a.template get<R>(F);
        st->am = a.template get<int>(F);
        st->inv2 = a.template get<int>(T);
        st->err = a.template get<int>(1);
        st->nck = nck;
        st->every = every;
        adj = std::move(st);
    }

    void adjoint_record(int nsteps, int every) override {
        finish_tail();
        if (grad_mode != MPS_GRAD_STANDARD)
            throw ApiError(MPS_ERR_UNSUPPORTED,
                           "the adjoint covers the default PrsGrdTrm only (MPS_GRAD_STANDARD)");
        if (motion_on)
            throw ApiError(MPS_ERR_UNSUPPORTED, "the adjoint needs static walls");
        if (nscene != 1)
            throw ApiError(MPS_ERR_UNSUPPORTED, "the adjoint runs on single-scene handles");
        if (nsteps <= 0 || every <= 0)
            throw ApiError(MPS_ERR_ARG, "nsteps and checkpoint_every must be positive");
        every = std::min(every, nsteps);
        const int nck = (nsteps + every - 1) / every;
        if (!adj || adj->nck != nck || adj->every != every) adj_alloc(nck, every);
        adj->nsteps = 0;
        for (int c = 0; c < nck; ++c) {
            snapshot(adj->ck[c]);
            step(std::min(every, nsteps - c * every));
        }
        snapshot(adj->ck[nck]);
        adj->nsteps = nsteps;
        adj->steps_end = steps;
        CK(cudaStreamSynchronize(stream));
    }

    // mirrors from the raw list into tape buffers, normals included
    void bin_mirrors_n(V4<R>* dpos, int* dslot, V4<R>* dnrm, int* dcs) {
        MirrorKeySrc<R, RN> ks{d_sc, nscene, dead(), U.pos, U.slot};
        MirrorGatherN<R> g{U.pos, U.slot, adj->unrm, dpos, dslot, dnrm};
        bin(ks, g, &cnt->mirror_raw, cap, dcs, L());
    }

    PassArgs<R, RN> tape_args(const V4<R>* mpos, const int* mslot, const int* mcs, int* nbl,
                              int* nbc, V4<R>* pre) {
        PassArgs<R, RN> a = args(M1, mcs1);
        a.m = MirrorView<R>{mcs, mpos, mslot};
        a.near_m = nullptr;  // the recorded mirror tables carry no near flags
        a.nb = nbl;
        a.nbcnt = nbc;
        a.tape_pre = pre;
        a.out.nrm = adj->unrm;
        return a;
    }

    // the first mirror generation of a replayed segment, as prepare_fused makes it
    void tape_prepare(const TapeStep<R>& t) {
        mkbkt(false);
        reset_raw();
        PassArgs<R, RN> a = tape_args(M1.pos, M1.slot, mcs1, nb, nbcnt, nullptr);
        k_gen_cull<R, RN, false, true><<<blocks(nF, block), block, 0, stream>>>(
            a, S.pos, S.prs, S.typ);
        KL();
        cull_raw();
        bin_mirrors_n(t.m1pos, t.m1slot, t.m1nrm, t.mcs1);
    }

    // fused_body with the recording kernels; `next` receives the next step's mirrors
    void tape_body(const TapeStep<R>& t, const TapeStep<R>* next) {
        const int ba = blk[MPS_K_PASS_A], bb = blk[MPS_K_PASS_B], bc = blk[MPS_K_PASS_C],
                  bg = blk[MPS_K_GEN];
        const size_t F = size_t(nF);
        auto cp = [&](void* d, const void* s, size_t bytes) {
            CK(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, stream));
        };
        cp(t.pid1, S.pid, sizeof(int) * F);
        cp(t.x1, S.pos, sizeof(V4<R>) * F);
        cp(t.v1, S.vel, sizeof(V4<R>) * F);
        PassArgs<R, RN> a = tape_args(t.m1pos, t.m1slot, t.mcs1, t.nbA, t.nA, t.up1);
        k_pass_a<R, RN, false, true><<<blocks(nF, ba), ba, 0, stream>>>(a);
        KL();
        bin_fluid(t_pos, t_vel, nullptr, S.prs, S.pav, S.pid, t_typ);
        a = tape_args(t.m1pos, t.m1slot, t.mcs1, t.nbB, t.nB, nullptr);
        // the second mirror generation beside pass B, as in fused_body (overlap bit 1); the
        // recorded copies after pass B read only arrays the generation reads too
        const bool fork = (overlap & 2) && !timing_on;
        if (fork) {
            CK(cudaEventRecord(ev_fork, stream));
            CK(cudaStreamWaitEvent(side, ev_fork, 0));
            OnStream o(this, side);
            reset_raw();
            k_gen_cull<R, RN, false, true><<<blocks(nF, bg), bg, 0, stream>>>(a, S.pos, nullptr,
                                                                                    S.typ);
            KL();
            cull_raw();
            bin_mirrors_n(t.m2pos, t.m2slot, t.m2nrm, t.mcs2);
            CK(cudaEventRecord(ev_join, side));
        }
        k_pass_b<R, RN, false><<<blocks(nF, bb), bb, 0, stream>>>(a);
        KL();
        cp(t.pid2, S.pid, sizeof(int) * F);
        cp(t.x2, S.pos, sizeof(V4<R>) * F);
        cp(t.u2, S.vel, sizeof(V4<R>) * F);
        cp(t.vv2, t_vel, sizeof(V4<R>) * F);
        cp(t.P2, t_prs, sizeof(R) * F);
        if (fork) {
            CK(cudaStreamWaitEvent(stream, ev_join, 0));
            k_mirror_prs<R><<<std::min(blocks(std::max(cap, 1), 256), 148 * 8), 256, 0, stream>>>(
                t.mcs2, dead(), t.m2pos, t_prs, nF);
            KL();
        } else {
            reset_raw();
            k_gen_cull<R, RN, false, true><<<blocks(nF, bg), bg, 0, stream>>>(a, S.pos, t_prs,
                                                                                    S.typ);
            KL();
            cull_raw();
            bin_mirrors_n(t.m2pos, t.m2slot, t.m2nrm, t.mcs2);
        }
        a = tape_args(t.m2pos, t.m2slot, t.mcs2, t.nbB, t.nB, t.vp2);
        k_pass_c<R, RN, false, true><<<blocks(nF, bc), bc, 0, stream>>>(a);
        KL();
        reset_raw();
        k_gen_cull<R, RN, false, true><<<blocks(nF, bg), bg, 0, stream>>>(a, t_pos, t_prs,
                                                                                t_typ);
        KL();
        cull_raw();
        bin_fluid(t_pos, t_vel, nullptr, t_prs, S.pav, S.pid, t_typ);
        if (next) bin_mirrors_n(next->m1pos, next->m1slot, next->m1nrm, next->mcs1);
        else bin_mirrors(M1, mcs1);
    }

    void back_step(const TapeStep<R>& t) {
        AdjState& s = *adj;
        AdjArgs<R, RN> A;
        A.sc = d_sc; A.nF = nF; A.nbK = nbK; A.t = t; A.wl = wall_view();
        A.lx = s.lx; A.lv = s.lv; A.lx_acc = s.lx_acc;
        A.lG = s.lG; A.lvv = s.lvv; A.lxs = s.lxs; A.lx_at = s.lx_at;
        A.lP = s.lP; A.lP_at = s.lP_at; A.pmin = s.pmin; A.am = s.am; A.inv2 = s.inv2;
        A.lxs_pid = s.lxs_pid; A.lu_pid = s.lu_pid;
        A.la = s.la; A.lxa = s.lxa; A.lva = s.lva;
        A.lkn = s.lkn; A.err = s.err;
        const int g = blocks(nF, 128);
        k_adj_c1<R, RN><<<g, 128, 0, stream>>>(A);
        KL();
        k_adj_c2<R, RN><<<g, 128, 0, stream>>>(A);
        KL();
        k_adj_b2<R, RN><<<g, 128, 0, stream>>>(A);
        KL();
        k_adj_a1<R, RN><<<g, 128, 0, stream>>>(A);
        KL();
        k_adj_a2<R, RN><<<g, 128, 0, stream>>>(A);
        KL();
        k_adj_fin<<<g, 128, 0, stream>>>(d_fluid_ids, nF, s.lx, s.lx_acc);
        KL();
    }

    void adjoint_backward(const double* lam_pos, const double* lam_vel, double* g_pos,
                          double* g_vel, double* g_nu) override {
        if (!adj || adj->nsteps == 0)
            throw ApiError(MPS_ERR_STATE, "no recorded rollout: call mps_adjoint_record first");
        if (adj->nbK != nbK)
            throw ApiError(MPS_ERR_STATE, "the neighbour-list capacity changed since the rollout "
                                          "was recorded");
        if (nF == 0) return;
        AdjState& s = *adj;
        const size_t T = size_t(nT);
        const int gT = blocks(nT, 256), gF = blocks(nF, 128);
        // adjoints of the final state, fluid entries only
        auto load = [&](const double* src, V4<double>* dst) {
            CK(cudaMemsetAsync(dst, 0, sizeof(V4<double>) * T, stream));
            if (!src) return;
            CK(cudaMemcpyAsync(s.stage, src, 3 * T * sizeof(double), cudaMemcpyDefault, stream));
            k_adj_in<<<gT, 256, 0, stream>>>(s.stage, nT, s.lxs_pid);
            KL();
            k_adj_pick<<<gF, 128, 0, stream>>>(d_fluid_ids, nF, s.lxs_pid, dst);
            KL();
        };
        load(lam_pos, s.lx);
        load(lam_vel, s.lv);
        CK(cudaMemsetAsync(s.lx_acc, 0, sizeof(V4<double>) * T, stream));
        CK(cudaMemsetAsync(s.lkn, 0, sizeof(double), stream));
        CK(cudaMemsetAsync(s.err, 0, sizeof(int), stream));
        invalidate_graph();
        for (int c = s.nck - 1; c >= 0; --c) {
            restore(s.ck[c]);
            const int ns = std::min(s.every, s.nsteps - c * s.every);
            tape_prepare(s.tape[0]);
            for (int k = 0; k < ns; ++k) tape_body(s.tape[k], k + 1 < ns ? &s.tape[k + 1] : nullptr);
            for (int k = ns - 1; k >= 0; --k) back_step(s.tape[k]);
        }
        auto out = [&](const V4<double>* src, double* dst) {
            if (!dst) return;
            k_adj_out<<<gT, 256, 0, stream>>>(src, nT, s.stage);
            KL();
            CK(cudaMemcpyAsync(dst, s.stage, 3 * T * sizeof(double), cudaMemcpyDefault, stream));
        };
        out(s.lx, g_pos);
        out(s.lv, g_vel);
        double lkn = 0;
        int err = 0;
        CK(cudaMemcpyAsync(&lkn, s.lkn, sizeof(double), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(&err, s.err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        // back to the end of the rollout
        restore(s.ck[s.nck]);
        steps = s.steps_end;
        CK(cudaStreamSynchronize(stream));
        if (err)
            throw ApiError(MPS_ERR_OVERFLOW,
                           std::to_string(err) + " neighbour list(s) of the recorded rollout exceeded "
                           "their capacity of " + std::to_string(nbK) +
                           "; the adjoint needs every list within capacity");
        // kn = knm_vsc / n0 (derive_scene), so d/d knm_vsc = d/d kn / n0
        if (g_nu) *g_nu = lkn / double(infos[0].n0);
    }

    void integrals(int scene, double out[6]) override {
        finish_tail();
        if (!lists_valid) mkbkt(acc_dirty);
        std::vector<double> init(6 * size_t(nscene), 0.0);
        for (int s = 0; s < nscene; ++s) init[6 * s + 4] = -1e300;
        CK(cudaMemcpyAsync(d_integ, init.data(), sizeof(double) * init.size(), cudaMemcpyHostToDevice,
                           stream));
        dim3 grid(std::min(blocks(std::max(nF, 1), 256), 148 * 4), nscene);
        k_integrals<R, RN><<<grid, 256, 0, stream>>>(d_sc, cs, S.pos, S.vel, S.typ, d_nbxyz, d_integ);
        KL();
        CK(cudaMemcpyAsync(init.data(), d_integ, sizeof(double) * init.size(), cudaMemcpyDeviceToHost,
                           stream));
        CK(cudaStreamSynchronize(stream));
        const double* v = init.data() + 6 * scene;
        double n = v[5];
        out[0] = n > 0 ? v[0] / n : 0;
        out[1] = n > 0 ? v[1] / n : 0;
        out[2] = n > 0 ? v[2] / n : 0;
        out[3] = v[3];
        out[4] = n > 0 ? v[4] : 0;
        out[5] = n;
    }
};

// one explicit instantiation per translation unit (mps_inst_*.cu)
SolverBase* make_solver_f32(int ns, const mps_params* p, const int32_t* c, const int8_t* t,
                            const void* pos, const void* vel, const void* nrm);
SolverBase* make_solver_f64(int ns, const mps_params* p, const int32_t* c, const int8_t* t,
                            const void* pos, const void* vel, const void* nrm);
SolverBase* make_solver_mix(int ns, const mps_params* p, const int32_t* c, const int8_t* t,
                            const void* pos, const void* vel, const void* nrm);

}  // namespace mps
