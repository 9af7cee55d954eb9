/*
 * mps_oracle.h -- C-ABI of the CPU oracle (TEST INFRASTRUCTURE, not the product).
 *
 * The oracle is a CPU restatement of the explicit MPS step of frsykzk/MPS_CUDA
 * (kernel.cu:307-1944), OpenMP over particles, templated on the arithmetic type. It keeps
 * the reference's data layout (arrays in particle-id order, NumMRR mirror slots per
 * particle) and runs the reference's per-particle loop bodies. It is used only by the
 * tests, by the `cpu_baseline` leg of bench.py and by bench.py's reference arm; the
 * product (mps_cuda_b200) never links or calls it.
 *
 * The parameter struct has the same field order as mps_params in include/mps_b200.h so
 * that callers can fill both from one record.
 */
#ifndef MPS_ORACLE_H
#define MPS_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_params {
    double pcl_dst, min[3], max[3], g[3], knm_vsc, col_rat, dst_lmt_rat, rho, snd, dt, umax,
        pmax;
    int32_t precision; /* 0 float, 1 double, 2 float state + double number density */
    int32_t reserved[7];
} oracle_params;

/* Dam-break scene description (same field order as mps_scene_desc): oracle_scene.cpp */
typedef struct oracle_scene_desc {
    double l0, tank[3];
    int32_t block[3], wall_mask;
    double jitter;
    uint64_t seed;
    double vel_sigma;
    uint64_t vel_seed;
    double origin[3];
} oracle_scene_desc;

/* particles of a dam-break scene; typ[n], pos/vel/nrm double SoA with stride cap */
int oracle_scene_dambreak_count(const oracle_scene_desc* d, int32_t* n_out);
int oracle_scene_dambreak(const oracle_scene_desc* d, int32_t cap, int8_t* typ, double* pos,
                          double* vel, double* nrm);
/* its parameters: domain = tank, SetPara's umax / Pmax along gravity on z */
int oracle_params_dambreak(const oracle_scene_desc* d, double snd, double dt, double knm_vsc,
                           double g_z, int32_t precision, oracle_params* p);

void* oracle_create(const oracle_params* p, int32_t n, const int8_t* typ, const void* pos,
                    const void* vel, const void* nrm);
void oracle_destroy(void* h);
int oracle_set_threads(int32_t n);
/* phase numbering is MPS_PHASE_* of include/mps_b200.h */
int oracle_phase(void* h, int32_t phase);
int oracle_step(void* h, int32_t nsteps);
/* PrsGrdTrm variant: 0 as compiled (kernel.cu:1651-1794), 1 the corrected-matrix #if 0
 * variant (kernel.cu:1435-1648) */
int oracle_set_gradient(void* h, int32_t mode);
/* prescribed rigid motion of the OBJ / OBJ2 walls, applied at the end of every step (the
 * same motion as mps_set_wall_motion) */
int oracle_set_wall_motion(void* h, int32_t type, const double* center, const double* axis,
                           double omega, const double* velocity);
int oracle_get_state(void* h, int8_t* typ, void* pos, void* vel, void* acc, void* prs,
                     void* pav);
int oracle_set_state(void* h, const int8_t* typ, const void* pos, const void* vel,
                     const void* acc, const void* prs, const void* pav);
int oracle_get_wall_flags(void* h, int8_t* wllse);
int oracle_set_wall_flags(void* h, const int8_t* wllse);
/* MRR slots in ascending slot order; pos is SoA with stride cap */
int oracle_get_mirrors(void* h, int32_t cap, int32_t* slot, void* pos, void* prs,
                       int32_t* n_out);
/* replace every mirror slot: slots not listed become GST */
int oracle_set_mirrors(void* h, int32_t n, const int32_t* slot, const void* pos,
                       const void* prs);
/* [n][11] table, columns MPS_DIAG_*; ndens[n] (real) */
int oracle_get_diag(void* h, int32_t* table, void* ndens);
/* out[0..]: n0, lmd, n0_grad, lmd_grad, numn0_grad, r, rp, db, dbinv, nbx, nby, nbz,
 * rlim2, col, prs_coef, minc xyz, maxc xyz */
int oracle_get_info(void* h, double* out);
/* out[6]: centroid xyz, sum |v|^2/2, max x, alive count (fluid) */
int oracle_get_integrals(void* h, double* out);

#ifdef __cplusplus
}
#endif
#endif
