// A ClcMPS-style driver (kernel.cu:1872-1943) ported to the facade: the same method calls
// in the same order, a state read-back at the output cadence, errors as exceptions.
#include <cstdio>
#include <vector>

#include "mps_b200.hpp"

int main() {
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
    } catch (const mps_b200::Error& e) {
        std::printf("%s\n", e.what());
        return e.status == MPS_ERR_NODEVICE ? 0 : 1;
    }
    return 0;
}
