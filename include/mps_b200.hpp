// mps_b200.hpp -- C++ facade over the C-ABI with the reference's method names.
//
// The reference's solver is `class MPS` (class.cuh:5-144) driven by ClcMPS
// (kernel.cu:1872-1943). This header keeps those method names so that a ClcMPS-style loop
// ports line by line; state comes in through the constructor (what RdDat + AlcBkt +
// SetPara did, kernel.cu:4-478) and goes out through DevicetoHost (kernel.cu:1847-1869).
// Every method throws mps_b200::Error carrying the C-ABI status instead of exit(1).
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "mps_b200.h"

namespace mps_b200 {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& where)
        : std::runtime_error(where + ": " + mps_status_string(s) + " (" + mps_last_error() + ")"),
          status(s) {}
};

inline void check(int s, const char* where) {
    if (s != MPS_OK) throw Error(s, where);
}

// Host copy of the state, SoA like the reference's areal3 members (const.cuh:67-71).
template <class real> struct State {
    std::vector<int8_t> Typ;
    std::vector<real> Pos, Vel, Acc;  // 3*n: x[n], y[n], z[n]
    std::vector<real> Prs, pav;
};

template <class real> class MPS {
   public:
    // typ/pos/vel/nrm as in initial.txt after RdDat: nrm is the inward normal (WLLVec)
    MPS(const mps_params& p, int n, const int8_t* typ, const real* pos, const real* vel,
        const real* nrm)
        : n_(n) {
        check(mps_create(&p, n, typ, pos, vel, nrm, &h_), "mps_create");
    }
    ~MPS() { mps_destroy(h_); }
    MPS(const MPS&) = delete;
    MPS& operator=(const MPS&) = delete;

    // class.cuh:8-28
    void MkBkt() { phase(MPS_PHASE_MKBKT); }
    void Surface_Edge() { phase(MPS_PHASE_SURFACE_EDGE); }
    void ResetMRR() { phase(MPS_PHASE_RESETMRR); }
    void GenMRR_nonslip() { phase(MPS_PHASE_GENMRR_NONSLIP); }
    void MkBkt_MRR() { phase(MPS_PHASE_MKBKT_MRR); }
    void VscTrm() { phase(MPS_PHASE_VSCTRM); }
    void UpPcl1() { phase(MPS_PHASE_UPPCL1); }
    void ChkCol() { phase(MPS_PHASE_CHKCOL); }
    void MkPrs() { phase(MPS_PHASE_MKPRS); }
    void PrsGrdTrm() { phase(MPS_PHASE_PRSGRDTRM); }
    void UpPcl2() { phase(MPS_PHASE_UPPCL2); }

    // n iterations of ClcMPS's loop body (kernel.cu:1904-1941), fused and stream-ordered
    void Step(int nsteps = 1) { check(mps_step(h_, nsteps), "mps_step"); }

    // kernel.cu:1847-1869
    void DevicetoHost(State<real>& s) {
        s.Typ.resize(n_);
        s.Pos.resize(3 * size_t(n_));
        s.Vel.resize(3 * size_t(n_));
        s.Acc.resize(3 * size_t(n_));
        s.Prs.resize(n_);
        s.pav.resize(n_);
        check(mps_get_state(h_, s.Typ.data(), s.Pos.data(), s.Vel.data(), s.Acc.data(),
                            s.Prs.data(), s.pav.data()),
              "mps_get_state");
    }

    mps_info Info(int scene = 0) {
        mps_info i;
        check(mps_get_info(h_, scene, &i), "mps_get_info");
        return i;
    }
    mps_counters Counters() {
        mps_counters c;
        check(mps_get_counters(h_, &c), "mps_get_counters");
        return c;
    }
    void SetStream(void* cuda_stream) { check(mps_set_stream(h_, cuda_stream), "mps_set_stream"); }
    void SetOption(int opt, int value) { check(mps_set_option(h_, opt, value), "mps_set_option"); }
    // MPS_GRAD_STANDARD (the compiled PrsGrdTrm) or MPS_GRAD_CORRECTED (its #if 0 variant)
    void SetGradient(int variant) { SetOption(MPS_OPT_GRADIENT, variant); }
    // prescribed rigid motion of the OBJ or OBJ2 walls (the declared rotating wall)
    void SetWallMotion(int type, const double center[3], const double axis[3], double omega,
                       const double velocity[3]) {
        check(mps_set_wall_motion(h_, type, center, axis, omega, velocity), "mps_set_wall_motion");
    }
    mps_handle* handle() { return h_; }

   private:
    void phase(int ph) { check(mps_phase(h_, ph), "mps_phase"); }
    mps_handle* h_ = nullptr;
    int n_;
};

// A case directory as RdDat reads it (MPS_physical.txt + initial.txt, kernel.cu:4-143) and
// the parameters SetPara derives (kernel.cu:396-415). pos/vel/nrm are SoA with stride n.
template <class real> struct Case {
    mps_physical phys;
    mps_params params;
    int n = 0;
    std::vector<int8_t> Typ;
    std::vector<real> Pos, Vel, Nrm;
};

template <class real> Case<real> RdDat(const std::string& dir, int precision) {
    Case<real> c;
    check(mps_read_physical((dir + "/MPS_physical.txt").c_str(), &c.phys), "mps_read_physical");
    const std::string init = dir + "/initial.txt";
    int32_t n = 0;
    mps_read_initial(init.c_str(), &c.phys, 0, nullptr, nullptr, nullptr, &n);  // sizing call
    std::vector<double> pos(3 * size_t(n)), nrm(3 * size_t(n));
    c.Typ.resize(n);
    check(mps_read_initial(init.c_str(), &c.phys, n, c.Typ.data(), pos.data(), nrm.data(), &n),
          "mps_read_initial");
    check(mps_params_from_physical(&c.phys, n, c.Typ.data(), pos.data(), precision, &c.params),
          "mps_params_from_physical");
    c.n = n;
    c.Pos.assign(pos.begin(), pos.end());
    c.Nrm.assign(nrm.begin(), nrm.end());
    c.Vel.assign(3 * size_t(n), real(0));
    return c;
}

// The reference's output files: WrtDatWLL when constructed, then WrtDat and WrtDat2
// (kernel.cu:279-304). WrtDat returns once the GPU has copied the state; a writer thread
// formats the CSV files. Close (or the destructor) waits for them; destroy it before the
// solver.
class Output {
   public:
    Output(mps_handle* h, const std::string& dir) {
        check(mps_output_open(h, dir.c_str(), &o_), "mps_output_open");
    }
    ~Output() {
        if (o_) mps_output_close(o_);
    }
    Output(const Output&) = delete;
    Output& operator=(const Output&) = delete;
    void WrtDat(int iF, double OPT_FQC) { check(mps_output_write(o_, iF, OPT_FQC), "mps_output_write"); }
    void WrtDat2() { check(mps_output_restart(o_), "mps_output_restart"); }
    void Close() {
        const int s = mps_output_close(o_);
        o_ = nullptr;
        check(s, "mps_output_close");
    }

   private:
    mps_output* o_ = nullptr;
};

}  // namespace mps_b200
