// mps_output.cu -- the reference's CSV output, written while the solver keeps stepping.
//
// WrtDat (kernel.cu:279-292) writes the fluid (output%05d.csv) and the mirrors
// (outputMRR%05d.csv) of the current state and then zeroes the time-summed pressure pav;
// WrtDatWLL (kernel.cu:295-299) writes the walls and their normals once; WrtDat2
// (kernel.cu:301-304) writes the fluid as a restart file (seitei.txt). Column layout and
// number format follow Output_vtk / Output_vtk2 (kernel.cu:161-276).
//
// The reference copies the whole state to the host and formats the files before its next
// step. Here mps_output_write snapshots the state into device staging on the solver's stream,
// waits only until the GPU reaches that snapshot, and returns: a side stream copies the
// staging to pinned host memory and a writer thread formats the files while the caller
// queues further steps. One snapshot is in flight at a time; the next write waits for it.
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mps_solver.cuh"

namespace mps {
int fail(int code, const std::string& msg);
}

namespace {

using mps::ApiError;

struct Pinned {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t n) {
        if (n <= bytes) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        if (cudaHostAlloc(&p, n, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            throw ApiError(MPS_ERR_NOMEM, "cudaHostAlloc of " + std::to_string(n) + " bytes failed");
        }
        bytes = n;
    }
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

}  // namespace

struct mps_output {
    mps::SolverBase* s = nullptr;  // the handle outlives the output set
    int dev = 0;
    std::string dir;
    int rsize = 4;  // bytes of the state type
    int n = 0, cap = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t snap = nullptr, copied = nullptr;
    mps::DevArena ar;
    // device staging
    void *d_pos, *d_vel, *d_prs, *d_pav, *d_mpos;
    int8_t* d_typ;
    int* d_mslot;
    // pinned host copies
    Pinned h_pos, h_vel, h_prs, h_pav, h_typ, h_mpos, h_mslot, h_count;
    // the writer thread's one job
    std::thread writer;
    std::mutex mu;
    std::condition_variable cv;
    bool pending = false, stop = false;
    int job_index = 0, job_mirrors = 0;
    double job_fqc = 1.0;
    std::string error;  // first I/O error, reported by the next call

    double val(const Pinned& b, size_t i) const {
        return rsize == 8 ? static_cast<const double*>(b.p)[i] : double(static_cast<const float*>(b.p)[i]);
    }
    std::string path(const char* name, int index) const {
        char buf[64];
        std::snprintf(buf, sizeof buf, name, index);
        return dir + "/" + buf;
    }
    void set_error(const std::string& e) {
        std::lock_guard<std::mutex> l(mu);
        if (error.empty()) error = e;
    }

    // Output_vtk(FLD, 0) and Output_vtk(MRR, 2) (kernel.cu:161-215)
    void format(int index, int nm, double fqc) {
        const size_t N = size_t(n);
        std::string p = path("output%05d.csv", index);
        if (FILE* f = std::fopen(p.c_str(), "w")) {
            std::fprintf(f, "Pos.x,Pos.y,Pos.z,Vel.x,Vel.y,Vel.z,Vel,Prs,pav\n");
            const int8_t* ty = static_cast<const int8_t*>(h_typ.p);
            for (size_t i = 0; i < N; ++i) {
                if (ty[i] != mps::kFLD) continue;
                double vx = val(h_vel, i), vy = val(h_vel, N + i), vz = val(h_vel, 2 * N + i), sp, pv;
                if (rsize == 8) {
                    sp = std::sqrt(vx * vx + vy * vy + vz * vz);
                    pv = val(h_pav, i) / fqc;
                } else {  // the reference's float arithmetic: sqrt(float), real / real
                    const float fx = float(vx), fy = float(vy), fz = float(vz);
                    sp = double(std::sqrt(fx * fx + fy * fy + fz * fz));
                    pv = double(float(val(h_pav, i)) / float(fqc));
                }
                std::fprintf(f, "%f,%f,%f,%f,%f,%f,%f,%f,%f\n", val(h_pos, i), val(h_pos, N + i),
                             val(h_pos, 2 * N + i), vx, vy, vz, sp, val(h_prs, i), pv);
            }
            if (std::fclose(f) != 0) set_error("write failed: " + p);
        } else {
            set_error("cannot create " + p);
        }
        // mirrors in slot order, as the reference walks its slots (kernel.cu:205-212)
        std::vector<int> order(nm);
        const int* sl = static_cast<const int*>(h_mslot.p);
        for (int k = 0; k < nm; ++k) order[k] = k;
        std::sort(order.begin(), order.end(), [&](int a, int b) { return sl[a] < sl[b]; });
        p = path("outputMRR%05d.csv", index);
        if (FILE* f = std::fopen(p.c_str(), "w")) {
            std::fprintf(f, "PosM.x,PosM.y,PosM.z,VelM,PrsM\n");
            for (int k : order) {
                if (sl[k] < 0) continue;
                const size_t q = size_t(k) * 4;  // V4: x, y, z, w = PrsM
                std::fprintf(f, "%f,%f,%f,%f,%f,\n", val(h_mpos, q), val(h_mpos, q + 1),
                             val(h_mpos, q + 2), 0.0, val(h_mpos, q + 3));
            }
            if (std::fclose(f) != 0) set_error("write failed: " + p);
        } else {
            set_error("cannot create " + p);
        }
    }

    void run() {
        std::unique_lock<std::mutex> l(mu);
        for (;;) {
            cv.wait(l, [&] { return pending || stop; });
            if (!pending) return;
            const int index = job_index, nm = job_mirrors;
            const double fqc = job_fqc;
            l.unlock();
            cudaError_t e = cudaEventSynchronize(copied);
            if (e != cudaSuccess) set_error(std::string("output copy: ") + cudaGetErrorString(e));
            else format(index, nm, fqc);
            l.lock();
            pending = false;
            cv.notify_all();
        }
    }

    void wait_idle() {
        std::unique_lock<std::mutex> l(mu);
        cv.wait(l, [&] { return !pending; });
    }

    int take_error() {
        std::lock_guard<std::mutex> l(mu);
        if (error.empty()) return MPS_OK;
        std::string e = error;
        error.clear();
        return mps::fail(MPS_ERR_ARG, e);
    }
};

namespace {

template <class F> int out_guard(mps_output* o, F&& f) {
    if (!o || !o->s) return mps::fail(MPS_ERR_ARG, "null output");
    try {
        if (cudaSetDevice(o->dev) != cudaSuccess) return mps::fail(MPS_ERR_CUDA, "cudaSetDevice failed");
        f(*o);
        return o->take_error();
    } catch (const ApiError& e) {
        return mps::fail(e.code, e.what());
    } catch (const std::exception& e) {
        return mps::fail(MPS_ERR_CUDA, e.what());
    }
}

}  // namespace

extern "C" {

int mps_output_open(mps_handle* h, const char* dir, mps_output** out) {
    if (!out) return mps::fail(MPS_ERR_ARG, "out is null");
    *out = nullptr;
    if (!h || !h->s || !dir) return mps::fail(MPS_ERR_ARG, "handle and dir must be given");
    auto* o = new mps_output();
    o->s = h->s.get();
    o->dev = o->s->dev;
    o->dir = dir;
    o->rsize = o->s->precision == MPS_F64 ? 8 : 4;
    o->n = o->s->nT;
    o->cap = o->s->cap;
    int rc = out_guard(o, [&](mps_output& q) {
        const size_t N = size_t(std::max(q.n, 1)), R = size_t(q.rsize);
        q.d_pos = q.ar.get<char>(3 * N * R);
        q.d_vel = q.ar.get<char>(3 * N * R);
        q.d_prs = q.ar.get<char>(N * R);
        q.d_pav = q.ar.get<char>(N * R);
        q.d_typ = q.ar.get<int8_t>(N);
        q.d_mpos = q.ar.get<char>(size_t(std::max(q.cap, 1)) * 4 * R);
        q.d_mslot = q.ar.get<int>(size_t(std::max(q.cap, 1)));
        q.h_pos.ensure(3 * N * R);
        q.h_vel.ensure(3 * N * R);
        q.h_prs.ensure(N * R);
        q.h_pav.ensure(N * R);
        q.h_typ.ensure(N);
        q.h_count.ensure(sizeof(int));
        if (cudaStreamCreateWithFlags(&q.side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&q.snap, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&q.copied, cudaEventDisableTiming) != cudaSuccess)
            throw ApiError(MPS_ERR_CUDA, "output stream or events");
        // WrtDatWLL (kernel.cu:295-299): walls and their normals, file index 0
        std::vector<int8_t> ty(N), se(N);
        std::vector<char> pos(3 * N * R), nrm(3 * N * R);
        q.s->get_state(ty.data(), pos.data(), nullptr, nullptr, nullptr, nullptr);
        q.s->get_wall_flags(se.data());
        q.s->get_wall_normals(nrm.data());
        auto v = [&](const std::vector<char>& b, size_t i) {
            return q.rsize == 8 ? reinterpret_cast<const double*>(b.data())[i]
                                : double(reinterpret_cast<const float*>(b.data())[i]);
        };
        const size_t n = size_t(q.n);
        std::string p = q.path("outputwall%05d.csv", 0);
        FILE* f = std::fopen(p.c_str(), "w");
        if (!f) throw ApiError(MPS_ERR_ARG, "cannot create " + p);
        std::fprintf(f, "Pos.x,Pos.y,Pos.z,Prs,pav,SE\n");
        for (size_t i = 0; i < n; ++i)
            if (ty[i] == mps::kWLL)
                std::fprintf(f, "%f,%f,%f,%f,%f,%d\n", v(pos, i), v(pos, n + i), v(pos, 2 * n + i),
                             0.0, 0.0, int(se[i]));
        if (std::fclose(f) != 0) throw ApiError(MPS_ERR_ARG, "write failed: " + p);
        p = q.path("outputWLLvec%05d.csv", 0);
        f = std::fopen(p.c_str(), "w");
        if (!f) throw ApiError(MPS_ERR_ARG, "cannot create " + p);
        std::fprintf(f, "PosM.x,PosM.y,PosM.z,vec.x,vec.y,vec.z\n");
        for (size_t i = 0; i < n; ++i)
            if (ty[i] == mps::kWLL)
                std::fprintf(f, "%f,%f,%f,%f,%f,%f\n", v(pos, i), v(pos, n + i), v(pos, 2 * n + i),
                             v(nrm, i), v(nrm, n + i), v(nrm, 2 * n + i));
        if (std::fclose(f) != 0) throw ApiError(MPS_ERR_ARG, "write failed: " + p);
        q.writer = std::thread([&q] { q.run(); });
    });
    if (rc != MPS_OK) {
        mps_output_close(o);
        return rc;
    }
    *out = o;
    return MPS_OK;
}

int mps_output_write(mps_output* o, int32_t index, double opt_fqc) {
    if (!(opt_fqc > 0)) return mps::fail(MPS_ERR_ARG, "opt_fqc (steps summed into pav) must be positive");
    return out_guard(o, [&](mps_output& q) {
        q.wait_idle();  // the staging and host buffers of the previous snapshot are free
        mps::SolverBase& s = *q.s;
        int* count = static_cast<int*>(q.h_count.p);
        s.output_snapshot(q.d_pos, q.d_vel, q.d_prs, q.d_pav, q.d_typ, q.d_mpos, q.d_mslot, count);
        CK(cudaEventRecord(q.snap, s.stream));
        CK(cudaEventSynchronize(q.snap));  // the GPU reached the snapshot: the mirror count is known
        const int nm = std::min(*count, q.cap);
        const size_t N = size_t(q.n), R = size_t(q.rsize);
        q.h_mpos.ensure(size_t(std::max(nm, 1)) * 4 * R);
        q.h_mslot.ensure(size_t(std::max(nm, 1)) * sizeof(int));
        CK(cudaMemcpyAsync(q.h_pos.p, q.d_pos, 3 * N * R, cudaMemcpyDeviceToHost, q.side));
        CK(cudaMemcpyAsync(q.h_vel.p, q.d_vel, 3 * N * R, cudaMemcpyDeviceToHost, q.side));
        CK(cudaMemcpyAsync(q.h_prs.p, q.d_prs, N * R, cudaMemcpyDeviceToHost, q.side));
        CK(cudaMemcpyAsync(q.h_pav.p, q.d_pav, N * R, cudaMemcpyDeviceToHost, q.side));
        CK(cudaMemcpyAsync(q.h_typ.p, q.d_typ, N, cudaMemcpyDeviceToHost, q.side));
        if (nm > 0) {
            CK(cudaMemcpyAsync(q.h_mpos.p, q.d_mpos, size_t(nm) * 4 * R, cudaMemcpyDeviceToHost, q.side));
            CK(cudaMemcpyAsync(q.h_mslot.p, q.d_mslot, size_t(nm) * sizeof(int), cudaMemcpyDeviceToHost,
                               q.side));
        }
        CK(cudaEventRecord(q.copied, q.side));
        std::lock_guard<std::mutex> l(q.mu);
        q.job_index = index;
        q.job_mirrors = nm;
        q.job_fqc = opt_fqc;
        q.pending = true;
        q.cv.notify_all();
    });
}

int mps_output_restart(mps_output* o) {
    return out_guard(o, [&](mps_output& q) {
        // Output_vtk2 (kernel.cu:251-276): the fluid as 'idx typ x y z 0 0 0 0'
        const size_t N = size_t(std::max(q.n, 1)), R = size_t(q.rsize), n = size_t(q.n);
        std::vector<int8_t> ty(N);
        std::vector<char> pos(3 * N * R);
        q.s->get_state(ty.data(), pos.data(), nullptr, nullptr, nullptr, nullptr);
        auto v = [&](size_t i) {
            return q.rsize == 8 ? reinterpret_cast<const double*>(pos.data())[i]
                                : double(reinterpret_cast<const float*>(pos.data())[i]);
        };
        std::string p = q.dir + "/seitei.txt";
        FILE* f = std::fopen(p.c_str(), "w");
        if (!f) throw ApiError(MPS_ERR_ARG, "cannot create " + p);
        int nf = 0;
        for (size_t i = 0; i < n; ++i) nf += ty[i] == mps::kFLD;
        std::fprintf(f, "%d\n", nf);
        int k = 0;
        for (size_t i = 0; i < n; ++i)
            if (ty[i] == mps::kFLD)
                std::fprintf(f, "%d %d %f %f %f %f %f %f %f\n", k++, int(ty[i]), v(i), v(n + i),
                             v(2 * n + i), 0.0, 0.0, 0.0, 0.0);
        if (std::fclose(f) != 0) throw ApiError(MPS_ERR_ARG, "write failed: " + p);
    });
}

int mps_output_close(mps_output* o) {
    if (!o) return MPS_OK;
    int rc = MPS_OK;
    if (o->writer.joinable()) {
        o->wait_idle();
        {
            std::lock_guard<std::mutex> l(o->mu);
            o->stop = true;
            o->cv.notify_all();
        }
        o->writer.join();
    }
    rc = o->take_error();
    cudaSetDevice(o->dev);
    if (o->side) cudaStreamDestroy(o->side);
    if (o->snap) cudaEventDestroy(o->snap);
    if (o->copied) cudaEventDestroy(o->copied);
    delete o;
    return rc;
}

}  // extern "C"
