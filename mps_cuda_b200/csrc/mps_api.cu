// mps_api.cu -- the C-ABI of include/mps_b200.h over the templated solver.
//
// One handle owns the device state of one or more scenes. The reference keeps that state
// in public members of `class MPS` (class.cuh:49-141) and drives it from ClcMPS
// (kernel.cu:1872-1943) with a blocking cudaDeviceSynchronize after every kernel; here the
// whole step is queued on one stream (optionally replayed as a CUDA graph) and nothing
// synchronises until the caller reads data back.
#include "mps_solver.cuh"

namespace mps {
thread_local std::string g_last_error;

namespace {
std::mutex g_tune_mu;
std::map<TuneKey, Tuned> g_tune;
}  // namespace
bool tuned_cache_get(const TuneKey& k, Tuned* out) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(k);
    if (it == g_tune.end()) return false;
    *out = it->second;
    return true;
}
void tuned_cache_put(const TuneKey& k, const Tuned& t) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[k] = t;
}
}  // namespace mps

// =========================================================================================
// C-ABI
// =========================================================================================
using mps::ApiError;
using mps::SolverBase;

namespace {
int fail(int code, const std::string& msg) {
    mps::g_last_error = msg;
    return code;
}

template <class F> int guarded(mps_handle* h, F&& f) {
    if (!h || !h->s) return fail(MPS_ERR_ARG, "null handle");
    try {
        cudaError_t e = cudaSetDevice(h->s->dev);
        if (e != cudaSuccess) return fail(MPS_ERR_CUDA, cudaGetErrorString(e));
        f(*h->s);
        return MPS_OK;
    } catch (const ApiError& e) {
        return fail(e.code, e.what());
    } catch (const std::exception& e) {
        return fail(MPS_ERR_CUDA, e.what());
    }
}

int check_params(const mps_params& p) {
    if (!(p.pcl_dst > 0) || !(p.dt > 0) || !(p.rho > 0) || !(p.snd >= 0))
        return fail(MPS_ERR_ARG, "pcl_dst, dt and rho must be positive, snd non-negative");
    for (int d = 0; d < 3; ++d)
        if (!(p.max[d] > p.min[d])) return fail(MPS_ERR_ARG, "domain max must exceed min");
    if (p.precision < 0 || p.precision > 2) return fail(MPS_ERR_ARG, "unknown precision");
    return MPS_OK;
}

// derived constants of a scene in its precision (host only); a grid too large for the
// int32 cell indices is reported here, before any device is touched
int derive_checked(const mps_params& p, mps_info* out) {
    mps_info tmp;
    if (!out) out = &tmp;
    try {
        if (p.precision == 1) {
            mps::SceneDev<double, double> sd;
            mps::derive_scene<double, double>(p, 0, 0, 0, 0, sd, *out);
        } else if (p.precision == 2) {
            mps::SceneDev<float, double> sd;
            mps::derive_scene<float, double>(p, 0, 0, 0, 0, sd, *out);
        } else {
            mps::SceneDev<float, float> sd;
            mps::derive_scene<float, float>(p, 0, 0, 0, 0, sd, *out);
        }
    } catch (const ApiError& e) {
        return fail(e.code, e.what());
    }
    return MPS_OK;
}
}  // namespace

extern "C" {

int mps_create_batch(int32_t nscenes, const mps_params* p, const int32_t* counts,
                     const int8_t* typ, const void* pos, const void* vel, const void* nrm,
                     mps_handle** out) {
    if (!out) return fail(MPS_ERR_ARG, "out is null");
    *out = nullptr;
    if (nscenes <= 0 || !p || !counts || !typ || !pos || !vel || !nrm)
        return fail(MPS_ERR_ARG, "null argument or no scenes");
    long long total = 0;
    for (int s = 0; s < nscenes; ++s) {
        int rc = check_params(p[s]);
        if (!rc) rc = derive_checked(p[s], nullptr);
        if (rc) return rc;
        if (p[s].precision != p[0].precision)
            return fail(MPS_ERR_ARG, "every scene of a batch must use the same precision");
        if (counts[s] < 0) return fail(MPS_ERR_ARG, "negative particle count");
        total += counts[s];
    }
    if (total * mps::kNumMRR > 2000000000LL) return fail(MPS_ERR_ARG, "too many particles");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MPS_ERR_NODEVICE, "no CUDA device");
    }
    auto* h = new mps_handle();
    try {
        if (p[0].precision == 1)
            h->s.reset(mps::make_solver_f64(nscenes, p, counts, typ, pos, vel, nrm));
        else if (p[0].precision == 2)
            h->s.reset(mps::make_solver_mix(nscenes, p, counts, typ, pos, vel, nrm));
        else
            h->s.reset(mps::make_solver_f32(nscenes, p, counts, typ, pos, vel, nrm));
    } catch (const ApiError& e) {
        delete h;
        return fail(e.code, e.what());
    } catch (const std::exception& e) {
        delete h;
        return fail(MPS_ERR_CUDA, e.what());
    }
    *out = h;
    return MPS_OK;
}

int mps_select_device(int32_t device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MPS_ERR_NODEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(MPS_ERR_ARG, "device index out of range");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(MPS_ERR_CUDA, cudaGetErrorString(e));
    return MPS_OK;
}

int mps_derive(const mps_params* p, mps_info* out) {
    if (!p || !out) return fail(MPS_ERR_ARG, "null argument");
    int rc = check_params(*p);
    if (rc) return rc;
    return derive_checked(*p, out);
}

int mps_create(const mps_params* p, int32_t n, const int8_t* typ, const void* pos,
               const void* vel, const void* nrm, mps_handle** out) {
    return mps_create_batch(1, p, &n, typ, pos, vel, nrm, out);
}

int mps_destroy(mps_handle* h) {
    if (!h) return MPS_OK;
    if (h->s) {
        cudaSetDevice(h->s->dev);
        cudaStreamSynchronize(h->s->stream);
    }
    delete h;
    return MPS_OK;
}

int mps_set_stream(mps_handle* h, void* stream) {
    return guarded(h, [&](SolverBase& s) {
        CK(cudaStreamSynchronize(s.stream));
        // NULL selects the handle's own stream again
        s.stream = stream ? static_cast<cudaStream_t>(stream) : s.own_stream;
        s.invalidate_graph();
    });
}

int mps_set_option(mps_handle* h, int32_t opt, int32_t value) {
    return guarded(h, [&](SolverBase& s) {
        switch (opt) {
            case MPS_OPT_DIAG: s.diag_on = value != 0; break;
            case MPS_OPT_GRAPH: s.graph_on = value != 0; s.invalidate_graph(); break;
            case MPS_OPT_BLOCK:
                if (value != 0 && (value < 32 || value > 128 || value % 32))
                    throw ApiError(MPS_ERR_ARG, "block must be 0 or a multiple of 32 in [32, 128]");
                s.block = value ? value : 128;
                for (int g : {MPS_K_PASS_A, MPS_K_PASS_B, MPS_K_PASS_C, MPS_K_GEN}) s.blk[g] = s.block;
                s.invalidate_graph();
                break;
            case MPS_OPT_CELL_SKIP: s.skip_opt = value != 0; s.invalidate_graph(); break;
            case MPS_OPT_TIMING: s.timing_on = value != 0; break;
            case MPS_OPT_LIST_CAPACITY:
                if (value < 0) throw ApiError(MPS_ERR_ARG, "list capacity must not be negative");
                s.set_list_capacity(value);
                break;
            case MPS_OPT_STAGING:
                if (value < MPS_STAGE_GLOBAL || value > MPS_STAGE_VELOCITIES)
                    throw ApiError(MPS_ERR_ARG, "staging must be one of MPS_STAGE_*");
                s.stage_mode = value;
                s.invalidate_graph();
                break;
            case MPS_OPT_CANDIDATE_BATCH:
                if (value != 0 && value != 2 && value != 4 && value != 8)
                    throw ApiError(MPS_ERR_ARG, "candidate batch must be 0, 2, 4 or 8");
                s.batch_a = value ? value : 4;
                s.invalidate_graph();
                break;
            case MPS_OPT_REGISTER_BOUND:
                if (value < 0 || value > 7)
                    throw ApiError(MPS_ERR_ARG, "register bound must lie in [0, 7]");
                s.reg_bound = value;
                s.invalidate_graph();
                break;
            case MPS_OPT_OVERLAP:
                if (value < 0 || value > 3) throw ApiError(MPS_ERR_ARG, "overlap must lie in [0, 3]");
                s.overlap = value;
                s.invalidate_graph();
                break;
            case MPS_OPT_STAGE_CAPACITY:
                if (value < 0 || value > (1 << 16))
                    throw ApiError(MPS_ERR_ARG, "stage capacity must lie in [0, 65536]");
                s.stage_cap = value;
                s.invalidate_graph();
                break;
            case MPS_OPT_GRADIENT:
                if (value != MPS_GRAD_STANDARD && value != MPS_GRAD_CORRECTED)
                    throw ApiError(MPS_ERR_ARG, "gradient must be MPS_GRAD_STANDARD or _CORRECTED");
                s.grad_mode = value;
                s.invalidate_graph();
                break;
            default: throw ApiError(MPS_ERR_ARG, "unknown option");
        }
    });
}

int mps_get_option(mps_handle* h, int32_t opt, int32_t* value) {
    if (!value) return fail(MPS_ERR_ARG, "null value");
    return guarded(h, [&](SolverBase& s) {
        switch (opt) {
            case MPS_OPT_DIAG: *value = s.diag_on; break;
            case MPS_OPT_GRAPH: *value = s.graph_on; break;
            case MPS_OPT_BLOCK: *value = s.blk[MPS_K_PASS_A]; break;
            case MPS_OPT_CELL_SKIP: *value = s.skip_opt; break;
            case MPS_OPT_TIMING: *value = s.timing_on; break;
            case MPS_OPT_GRADIENT: *value = s.grad_mode; break;
            case MPS_OPT_LIST_CAPACITY: *value = s.list_capacity(); break;
            case MPS_OPT_STAGING: *value = s.stage_mode; break;
            case MPS_OPT_STAGE_CAPACITY: *value = s.stage_cap; break;
            case MPS_OPT_CANDIDATE_BATCH: *value = s.batch_a; break;
            case MPS_OPT_REGISTER_BOUND: *value = s.reg_bound; break;
            case MPS_OPT_OVERLAP: *value = s.overlap; break;
            default: throw ApiError(MPS_ERR_ARG, "unknown option");
        }
    });
}

int mps_set_wall_motion(mps_handle* h, int32_t type, const double center[3],
                        const double axis[3], double omega, const double velocity[3]) {
    return guarded(h, [&](SolverBase& s) { s.set_wall_motion(type, center, axis, omega, velocity); });
}

int mps_synchronize(mps_handle* h) {
    return guarded(h, [&](SolverBase& s) { CK(cudaStreamSynchronize(s.stream)); });
}

int mps_step(mps_handle* h, int32_t nsteps) {
    if (nsteps < 0) return fail(MPS_ERR_ARG, "negative step count");
    return guarded(h, [&](SolverBase& s) { s.step(nsteps); });
}

int mps_phase(mps_handle* h, int32_t phase) {
    return guarded(h, [&](SolverBase& s) { s.phase(phase); });
}

int mps_get_info(mps_handle* h, int32_t scene, mps_info* out) {
    return guarded(h, [&](SolverBase& s) {
        if (!out || scene < 0 || scene >= s.nscene) throw ApiError(MPS_ERR_ARG, "bad scene");
        *out = s.infos[scene];
        out->n_particles = s.counts[scene];
        out->n_fluid = s.nF;
        out->n_wall = s.nW;
    });
}

int mps_get_state(mps_handle* h, int8_t* typ, void* pos, void* vel, void* acc, void* prs,
                  void* pav) {
    return guarded(h, [&](SolverBase& s) { s.get_state(typ, pos, vel, acc, prs, pav); });
}

int mps_set_state(mps_handle* h, const int8_t* typ, const void* pos, const void* vel,
                  const void* acc, const void* prs, const void* pav) {
    return guarded(h, [&](SolverBase& s) { s.set_state(typ, pos, vel, acc, prs, pav); });
}

int mps_get_wall_flags(mps_handle* h, int8_t* wllse) {
    if (!wllse) return fail(MPS_ERR_ARG, "null buffer");
    return guarded(h, [&](SolverBase& s) { s.get_wall_flags(wllse); });
}

int mps_get_mirrors(mps_handle* h, int32_t which, int32_t cap, int32_t* slot, void* pos,
                    void* prs, int32_t* n_out) {
    if (which < 0 || which > 2 || cap < 0) return fail(MPS_ERR_ARG, "bad mirror request");
    return guarded(h, [&](SolverBase& s) {
        int n = s.get_mirrors(which, cap, slot, pos, prs);
        if (n_out) *n_out = n;
    });
}

int mps_get_diag(mps_handle* h, int32_t* table, void* ndens) {
    return guarded(h, [&](SolverBase& s) { s.get_diag(table, ndens); });
}

int mps_get_counters(mps_handle* h, mps_counters* out) {
    if (!out) return fail(MPS_ERR_ARG, "null buffer");
    return guarded(h, [&](SolverBase& s) { s.get_counters(out); });
}

int mps_get_work(mps_handle* h, mps_work* out) {
    if (!out) return fail(MPS_ERR_ARG, "null buffer");
    return guarded(h, [&](SolverBase& s) { s.get_work(out); });
}

int mps_get_timing(mps_handle* h, int32_t kernel, double* total_ms, int64_t* launches,
                   int32_t reset) {
    if (kernel < 0 || kernel >= MPS_K_COUNT) return fail(MPS_ERR_ARG, "unknown kernel group");
    return guarded(h, [&](SolverBase& s) {
        long long n = 0;
        s.timing(kernel, total_ms, &n, reset != 0);
        if (launches) *launches = n;
    });
}

int mps_adjoint_record(mps_handle* h, int32_t nsteps, int32_t checkpoint_every) {
    if (nsteps <= 0 || checkpoint_every <= 0)
        return fail(MPS_ERR_ARG, "nsteps and checkpoint_every must be positive");
    return guarded(h, [&](SolverBase& s) { s.adjoint_record(nsteps, checkpoint_every); });
}

int mps_adjoint_backward(mps_handle* h, const double* lam_pos, const double* lam_vel,
                         double* grad_pos0, double* grad_vel0, double* grad_nu) {
    return guarded(h, [&](SolverBase& s) {
        s.adjoint_backward(lam_pos, lam_vel, grad_pos0, grad_vel0, grad_nu);
    });
}

int mps_autotune(mps_handle* h, int32_t trial_steps, int32_t* chosen) {
    if (trial_steps <= 0) return fail(MPS_ERR_ARG, "trial_steps must be positive");
    return guarded(h, [&](SolverBase& s) { s.autotune(trial_steps, chosen); });
}

int mps_get_integrals(mps_handle* h, int32_t scene, double out[6]) {
    return guarded(h, [&](SolverBase& s) {
        if (!out || scene < 0 || scene >= s.nscene) throw ApiError(MPS_ERR_ARG, "bad scene");
        s.integrals(scene, out);
    });
}

const char* mps_status_string(int32_t st) {
    switch (st) {
        case MPS_OK: return "ok";
        case MPS_ERR_ARG: return "invalid argument";
        case MPS_ERR_CUDA: return "CUDA error";
        case MPS_ERR_NOMEM: return "out of memory";
        case MPS_ERR_STATE: return "invalid state";
        case MPS_ERR_OVERFLOW: return "capacity exceeded";
        case MPS_ERR_TIMEOUT: return "device wait timed out";
        case MPS_ERR_UNSUPPORTED: return "unsupported";
        case MPS_ERR_NODEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* mps_last_error(void) { return mps::g_last_error.c_str(); }

}  // extern "C"
