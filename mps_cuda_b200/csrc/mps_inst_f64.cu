// mps_inst_f64.cu -- instantiation of the solver for double state / double number density.
#include "mps_solver.cuh"

namespace mps {

SolverBase* make_solver_f64(int ns, const mps_params* p, const int32_t* c, const int8_t* t,
                            const void* pos, const void* vel, const void* nrm) {
    auto* s = new Solver<double, double>();
    try {
        s->init(ns, p, c, t, static_cast<const double*>(pos), static_cast<const double*>(vel),
                static_cast<const double*>(nrm));
    } catch (...) {
        delete s;
        throw;
    }
    return s;
}

}  // namespace mps
