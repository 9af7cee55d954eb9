// mps_inst_f32.cu -- instantiation of the solver for float state / float number density.
#include "mps_solver.cuh"

namespace mps {

SolverBase* make_solver_f32(int ns, const mps_params* p, const int32_t* c, const int8_t* t,
                            const void* pos, const void* vel, const void* nrm) {
    auto* s = new Solver<float, float>();
    try {
        s->init(ns, p, c, t, static_cast<const float*>(pos), static_cast<const float*>(vel),
                static_cast<const float*>(nrm));
    } catch (...) {
        delete s;
        throw;
    }
    return s;
}

}  // namespace mps
