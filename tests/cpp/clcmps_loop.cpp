// A ClcMPS-style driver (kernel.cu:1872-1943) ported to the facade: the same method calls
// in the same order, a state read-back at the output cadence, errors as exceptions.
#include <cstdio>
#include <filesystem>
#include <string>
#include <vector>

#include "mps_b200.hpp"

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    mps_scene_desc d = {};
    d.l0 = 0.02;
    d.tank[0] = 0.4; d.tank[1] = 0.2; d.tank[2] = 0.4;
    d.block[0] = 8; d.block[1] = 6; d.block[2] = 10;
    d.wall_mask = 0x1f;
    d.jitter = 0.01;
    int32_t n = 0;
    if (mps_scene_dambreak_count(&d, &n) != MPS_OK) return 2;
    std::vector<int8_t> typ(n);
    std::vector<double> pos(3 * n), vel(3 * n), nrm(3 * n);
    mps_scene_dambreak(&d, n, typ.data(), pos.data(), vel.data(), nrm.data(), &n);
    mps_params p;
    mps_params_dambreak(&d, 20.0, 2e-4, 1e-6, -9.81, MPS_F64, &p);
    // the same scene as a case directory, read back as RdDat reads it (no GPU needed)
    mps_physical ph = {};
    for (int k = 0; k < 3; ++k) { ph.max[k] = d.tank[k]; }
    ph.g[2] = -9.81; ph.fin_tim = 1.0; ph.output_time = 0.01; ph.mach = 0.1; ph.courant = 0.2;
    ph.col_rat = 0.2; ph.dst_lmt_rat = 0.9; ph.knm_vsc = 1e-6; ph.pcl_dst = d.l0;
    if (mps_write_physical((dir + "/MPS_physical.txt").c_str(), &ph) != MPS_OK ||
        mps_write_initial((dir + "/initial.txt").c_str(), n, typ.data(), pos.data(), nrm.data()) != MPS_OK)
        return 3;
    auto cs = mps_b200::RdDat<double>(dir, MPS_F64);
    if (cs.n != n || cs.Typ != typ || cs.Pos[0] != double(float(pos[0])) || !(cs.params.dt > 0))
        return 4;
    std::printf("case: %d particles, dt %g\n", cs.n, cs.params.dt);
    try {
        mps_b200::MPS<double> obj(p, n, typ.data(), pos.data(), vel.data(), nrm.data());
        mps_b200::State<double> st;
        for (int it = 0; it < 10; ++it) {
            obj.MkBkt();
            obj.ResetMRR(); obj.GenMRR_nonslip(); obj.MkBkt_MRR();
            obj.VscTrm();
            obj.UpPcl1();
            obj.MkBkt();
            obj.ChkCol();
            obj.MkBkt();
            obj.MkPrs();
            obj.ResetMRR(); obj.GenMRR_nonslip(); obj.MkBkt_MRR();
            obj.PrsGrdTrm();
            obj.UpPcl2();
        }
        obj.Step(10);  // the same loop body, fused
        obj.DevicetoHost(st);
        std::printf("alive %d\n", obj.Counters().n_fluid_alive);
        // the reference's #if 0 PrsGrdTrm for two steps, then the output files
        obj.SetGradient(MPS_GRAD_CORRECTED);
        obj.Step(2);
        obj.SetGradient(MPS_GRAD_STANDARD);
        std::filesystem::create_directories(dir + "/out");
        mps_b200::Output out(obj.handle(), dir + "/out");
        out.WrtDat(1, 2.0);
        out.WrtDat2();
        out.Close();
        if (!std::filesystem::exists(dir + "/out/output00001.csv")) return 5;
    } catch (const mps_b200::Error& e) {
        std::printf("%s\n", e.what());
        return e.status == MPS_ERR_NODEVICE ? 0 : 1;
    }
    return 0;
}
