/*
 * mps_b200.h -- C-ABI of the B200-native explicit MPS solver.
 *
 * This is the drop-in boundary for the explicit MPS time step of frsykzk/MPS_CUDA.
 * The reference exposes its solver only as `class MPS` (class.cuh:5-144): argument-less
 * methods operating on public members, device buffers allocated with cudaMalloc, errors
 * reported through `CHECK` -> exit(1) (const.cuh:87-95). This header replaces that
 * surface with a handle-based C-ABI: plain pointers and sizes, every call returns an
 * `int` status code (MPS_OK on success), nothing calls exit().
 *
 * Layout conventions
 *  - Particle arrays are indexed by particle id (the input order, = the reference's
 *    index `i` after RdDat, kernel.cu:110-131). Vectors are SoA: a `pos` buffer holds
 *    x[0..n), y[0..n), z[0..n) back to back (the reference's areal3, const.cuh:67-71).
 *  - `real` buffers are float for MPS_F32 / MPS_F32_N64 handles and double for MPS_F64.
 *  - Wall normals are the reference's WLLVec: unit vectors pointing INTO the fluid
 *    (RdDat negates the file normal, kernel.cu:127-128).
 *  - Host buffers are only borrowed for the duration of a call; device buffers are owned
 *    by the handle.
 *  - A handle is not thread-safe: use one handle per host thread. Work is queued on the
 *    handle's stream (mps_set_stream); calls that return host data synchronise it.
 */
#ifndef MPS_B200_H
#define MPS_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace CHECK -> exit(1), const.cuh:87-95) ---------------------- */
enum {
    MPS_OK = 0,
    MPS_ERR_ARG = 1,         /* invalid argument / inconsistent sizes                 */
    MPS_ERR_CUDA = 2,        /* a CUDA runtime call failed (see mps_last_error)        */
    MPS_ERR_NOMEM = 3,       /* device or host allocation failed                       */
    MPS_ERR_STATE = 4,       /* call not valid in the handle's current state           */
    MPS_ERR_OVERFLOW = 5,    /* a fixed capacity was exceeded (mirror slots, scratch)  */
    MPS_ERR_TIMEOUT = 6,     /* a bounded device-side wait ran out                     */
    MPS_ERR_UNSUPPORTED = 7, /* option not available in this build                     */
    MPS_ERR_NODEVICE = 8     /* no CUDA device                                         */
};

/* ---- particle types (const.cuh:28-33) and wall flags (const.cuh:35-36) -------------- */
enum { MPS_GST = -1, MPS_FLD = 0, MPS_WLL = 1, MPS_OBJ = 2, MPS_OBJ2 = 3, MPS_MRR = 4 };
enum { MPS_SURFACE = 0, MPS_EDGE = 1 };

/* maximum mirror particles generated from one fluid particle (const.cuh:50) */
#define MPS_NUM_MRR 10

/* ---- arithmetic of a handle (`typedef float real`, const.cuh:52-53) ----------------- */
enum {
    MPS_F32 = 0,     /* float state, float number density (the reference's typedef)  */
    MPS_F64 = 1,     /* double state (the commented `typedef double real`)            */
    MPS_F32_N64 = 2  /* float state, number density accumulated in double             */
};

/*
 * Physical parameters of one scene. Mirrors MPS_physical.txt (kernel.cu:12-22) plus the
 * values SetPara derives from it (kernel.cu:398-415) that are taken explicitly here:
 *  - `snd`, `dt`, `umax`, `pmax` are inputs. SetPara derives them from the fluid height
 *    along y and G.y (kernel.cu:399-415), which is degenerate when gravity points along z
 *    (umax = 0, dt = inf, Pmax = 0). mps_params_dambreak() fills them with
 *    umax = sqrt(2|g|H), pmax = rho |g| H for H the fluid height along gravity.
 *  - Prs_coef = snd^2 / n0_grad (kernel.cu:409) and every lattice constant are derived
 *    inside the library exactly as SetPara does (kernel.cu:336-373).
 */
typedef struct mps_params {
    double pcl_dst;      /* PCL_DST: particle spacing l0 [m]                    (item 17) */
    double min[3];       /* domain minimum before the 3.1*l0 padding            (items 1-3) */
    double max[3];       /* domain maximum before the 3.1*l0 padding            (items 4-6) */
    double g[3];         /* gravity G [m/s^2]                                   (items 7-9) */
    double knm_vsc;      /* KNM_VSC: kinematic viscosity [m^2/s]                (item 16) */
    double col_rat;      /* COL_RAT: collision restitution, COL = 1 + COL_RAT   (item 14) */
    double dst_lmt_rat;  /* DST_LMT_RAT: rlim = DST_LMT_RAT * l0                (item 15) */
    double rho;          /* particle density Dns of every type (const.cuh:38-41, kernel.cu:379-383) */
    double snd;          /* SND: sound speed [m/s]                                        */
    double dt;           /* time step [s]                                                 */
    double umax;         /* speed clamp in ChkPcl (kernel.cu:493)                          */
    double pmax;         /* pressure clamp in MkPrs (kernel.cu:1398)                       */
    int32_t precision;   /* MPS_F32 / MPS_F64 / MPS_F32_N64                               */
    int32_t reserved[7]; /* zero                                                          */
} mps_params;

/* Derived constants of a scene, as SetPara / AlcBkt compute them (kernel.cu:307-373). */
typedef struct mps_info {
    int32_t n_particles, n_fluid, n_wall;      /* nP, non-wall (FLD/GST), WLL/OBJ/OBJ2 */
    int32_t nbx, nby, nbz, nbxyz;              /* bucket grid (kernel.cu:317-322)       */
    double r, rp, db, dbinv;                   /* radii and bucket width (kernel.cu:309-315) */
    double n0, lmd, n0_grad, lmd_grad;         /* lattice sums (kernel.cu:341-365)      */
    int32_t numn0_grad, pad0;                  /* neighbour count of n0_grad            */
    double rlim2, col, prs_coef, pmax, umax, dt, snd;
    double minc[3], maxc[3];                   /* padded domain (kernel.cu:26-31)       */
} mps_info;

/* Device-side counters (host-side failure detection; nothing here traps the GPU). */
typedef struct mps_counters {
    int64_t steps;                 /* completed time steps                                  */
    int32_t n_fluid_alive;         /* FLD particles                                         */
    int32_t n_deleted;             /* GST particles among the non-wall particles            */
    int32_t n_mirror_1;            /* mirrors alive after the first generation of the step  */
    int32_t n_mirror_2;            /* mirrors alive after the second generation             */
    int32_t err_mirror_slot;       /* corner mirror found no free slot (kernel.cu:868-874)  */
    int32_t err_mirror_capacity;   /* mirror buffer full                                    */
    int32_t err_cell_range;        /* a bucket index left the grid and was clamped          */
    int32_t err_nan;               /* non-finite position met in a bucket build             */
    int32_t reserved0;
    int64_t kernel_launches;       /* kernels this handle launched (graph replays included) */
    int32_t stage_blocks;          /* with MPS_OPT_DIAG and staging: blocks of VscTrm that
                                      walked shared memory (cumulative)                     */
    int32_t unstaged_blocks;       /* ... and blocks whose neighbourhood did not fit        */
} mps_counters;

/* Per-particle diagnostic counters (mps_get_diag), column order of the int32 table. */
enum {
    MPS_DIAG_CELL = 0,      /* bucket index ib (kernel.cu:521-524), -1 for GST          */
    MPS_DIAG_VSC_F = 1,     /* VscTrm fluid neighbours, dist <= r      (kernel.cu:1057) */
    MPS_DIAG_VSC_M = 2,     /* VscTrm mirror neighbours                (kernel.cu:1092) */
    MPS_DIAG_COL_F = 3,     /* ChkCol fluid, dist2 < rlim2             (kernel.cu:1211) */
    MPS_DIAG_COL_W = 4,     /* ChkCol walls, dist2 < (0.45 l0)^2       (kernel.cu:1228) */
    MPS_DIAG_COL_M = 5,     /* ChkCol mirrors                          (kernel.cu:1261) */
    MPS_DIAG_PRS_F = 6,     /* MkPrs fluid, dist < rp                  (kernel.cu:1346) */
    MPS_DIAG_PRS_M = 7,     /* MkPrs mirrors                           (kernel.cu:1376) */
    MPS_DIAG_GRD_F = 8,     /* PrsGrdTrm fluid, dist2 < rp2            (kernel.cu:1730) */
    MPS_DIAG_GRD_M = 9,     /* PrsGrdTrm mirrors (j != i)              (kernel.cu:1768) */
    MPS_DIAG_GEN_W = 10,    /* GenMRR walls, dist2 <= r2               (kernel.cu:753)  */
    MPS_DIAG_NCOL = 11
};

/* Steps of the reference's time loop, one per `class MPS` method (class.cuh:8-28). */
enum {
    MPS_PHASE_MKBKT = 0,          /* MPS::MkBkt          kernel.cu:532-550  */
    MPS_PHASE_SURFACE_EDGE = 1,   /* MPS::Surface_Edge   kernel.cu:671-686  */
    MPS_PHASE_RESETMRR = 2,       /* MPS::ResetMRR       kernel.cu:704-717  */
    MPS_PHASE_GENMRR_NONSLIP = 3, /* MPS::GenMRR_nonslip kernel.cu:896-911  */
    MPS_PHASE_MKBKT_MRR = 4,      /* MPS::MkBkt_MRR      kernel.cu:987-1010 */
    MPS_PHASE_VSCTRM = 5,         /* MPS::VscTrm         kernel.cu:1122-1135 */
    MPS_PHASE_UPPCL1 = 6,         /* MPS::UpPcl1         kernel.cu:1152-1165 */
    MPS_PHASE_CHKCOL = 7,         /* MPS::ChkCol         kernel.cu:1289-1303 */
    MPS_PHASE_MKPRS = 8,          /* MPS::MkPrs          kernel.cu:1414-1427 */
    MPS_PHASE_PRSGRDTRM = 9,      /* MPS::PrsGrdTrm      kernel.cu:1798-1812 */
    MPS_PHASE_UPPCL2 = 10,        /* MPS::UpPcl2         kernel.cu:1831-1844 */
    MPS_PHASE_COUNT = 11
};

/* Handle options (mps_set_option). */
enum {
    MPS_OPT_DIAG = 0,        /* 1: record per-particle neighbour counts (slower)        */
    MPS_OPT_GRAPH = 1,       /* 1: replay mps_step through a captured CUDA graph        */
    MPS_OPT_BLOCK = 2,       /* threads per block of the neighbour passes (0 = tuned)   */
    MPS_OPT_CELL_SKIP = 3,   /* 1: skip bucket rows outside the radius (default 1)      */
    MPS_OPT_TIMING = 4,      /* 1: time every kernel group of mps_step with CUDA events
                                on the handle's stream (steps then run without a graph) */
    MPS_OPT_GRADIENT = 5,    /* PrsGrdTrm variant, MPS_GRAD_* (default STANDARD)        */
    MPS_OPT_LIST_CAPACITY = 6, /* neighbour-list entries kept per particle between ChkCol/
                                MkPrs and PrsGrdTrm: 0 or above 160 = 160 (the default).
                                A particle with more neighbours walks its fine cells again
                                instead, with the same result; lower values exercise that
                                path. Changing it voids a recorded adjoint rollout.       */
    MPS_OPT_STAGING = 7,     /* where VscTrm's candidate walk reads: MPS_STAGE_*         */
    MPS_OPT_STAGE_CAPACITY = 8, /* candidates a block may stage in shared memory (0 = the
                                default); a block whose neighbourhood holds more walks
                                global memory. Results never depend on it.               */
    MPS_OPT_CANDIDATE_BATCH = 9, /* VscTrm's candidates loaded together per particle: 2, 4
                                or 8 (0 = 4). Results never depend on it.                */
    MPS_OPT_REGISTER_BOUND = 10, /* bit 0: ChkCol/MkPrs, bit 1: PrsGrdTrm, bit 2: VscTrm
                                (walking global memory) at their alternate register bound
                                per thread (more or fewer resident blocks per SM; 0 = all
                                at the default). Results never depend on it.              */
    MPS_OPT_OVERLAP = 11     /* work on a second stream of the handle, bit 0: at the end
                                of a step the fluid bucket build beside the next step's
                                mirror generation; bit 1: the step's second mirror
                                generation (positions, cull, buckets) beside ChkCol/MkPrs,
                                its pressures filled in after them. 3 (both) is the
                                default, 0 one stream. Steps timed with MPS_OPT_TIMING
                                always use one stream. Results never depend on it.       */
};

/* MPS_OPT_STAGING. GLOBAL: each particle walks its fine cells through L1. POSITIONS: a block
 * first copies its particles' neighbourhood (the fine rows their walks reach) into shared
 * memory and walks it there. VELOCITIES: also the candidates' velocities. The candidates
 * and their order are the same in all three, so results are identical. */
enum { MPS_STAGE_GLOBAL = 0, MPS_STAGE_POSITIONS = 1, MPS_STAGE_VELOCITIES = 2 };

/* PrsGrdTrm variants (MPS_OPT_GRADIENT). STANDARD is the kernel the reference compiles
 * (kernel.cu:1651-1794). CORRECTED is its `#if 0` alternative (kernel.cu:1435-1648): the
 * moment matrix M = sum w r r^T / n0_grad of the fluid and mirror neighbours inside rp is
 * inverted and a = -1/rho M^-1 sum w (P_j - P_min) r / n0_grad. As in the reference, a
 * particle whose M is all zero keeps ChkCol's velocity as its acceleration, and a singular M
 * gives non-finite values, which ChkPcl deletes. The adjoint supports STANDARD only. */
enum { MPS_GRAD_STANDARD = 0, MPS_GRAD_CORRECTED = 1 };

/* Kernel groups reported by mps_get_timing. */
enum {
    MPS_K_PASS_A = 0,       /* VscTrm + UpPcl1                                   */
    MPS_K_PASS_B = 1,       /* ChkCol + MkPrs                                    */
    MPS_K_PASS_C = 2,       /* PrsGrdTrm + UpPcl2                                */
    MPS_K_GEN = 3,          /* GenMRR_nonslip + MRRinout (both generations)      */
    MPS_K_BIN_FLUID = 4,    /* fluid bucket builds (MkBkt)                       */
    MPS_K_BIN_MIRROR = 5,   /* mirror bucket builds (MkBkt_MRR)                  */
    MPS_K_COUNT = 6
};

typedef struct mps_handle mps_handle;

/* ---- scene set-up ----------------------------------------------------------------- */

/*
 * Dam-break scene: a rectangular tank [0,L]^3 with single-layer walls on the faces
 * selected by `wall_mask` (bit 0: x=0, 1: x=Lx, 2: y=0, 3: y=Ly, 4: z=0, 5: z=Lz), wall
 * particles at in-plane positions ((p+1/2)l0, (q+1/2)l0) of each face, and a fluid block
 * of nx*ny*nz particles at ((i+1/2)l0, (j+1/2)l0, (k+1/2)l0) + jitter.
 * Replaces the scene the reference reads from initial.txt (kernel.cu:59-141).
 */
typedef struct mps_scene_desc {
    double l0;                  /* spacing                                              */
    double tank[3];             /* tank extent                                          */
    int32_t block[3];           /* fluid particles along x, y, z                        */
    int32_t wall_mask;          /* faces with walls (0x1f = open top)                   */
    double jitter;              /* uniform jitter half-width as a fraction of l0        */
    uint64_t seed;              /* mt19937_64 seed of the jitter                        */
    double vel_sigma;           /* N(0, vel_sigma) initial velocity per component       */
    uint64_t vel_seed;          /* mt19937_64 seed of the velocities                    */
    double origin[3];           /* offset added to every position                       */
} mps_scene_desc;

/* Number of particles the scene will hold. */
int mps_scene_dambreak_count(const mps_scene_desc* d, int32_t* n_out);
/* Fill caller buffers (capacity >= count): typ[n], pos/vel/nrm as double SoA 3*n. */
int mps_scene_dambreak(const mps_scene_desc* d, int32_t cap, int8_t* typ, double* pos,
                       double* vel, double* nrm, int32_t* n_out);
/* Fill `p` for a dam break: domain = tank, umax = sqrt(2|g|H), pmax = rho|g|H. */
int mps_params_dambreak(const mps_scene_desc* d, double snd, double dt, double knm_vsc,
                        double g_z, int32_t precision, mps_params* p);

/*
 * Derived constants of one scene without creating a solver (host only, no GPU needed):
 * the values AlcBkt and SetPara compute (kernel.cu:307-373). n_particles/n_fluid/n_wall
 * are left zero.
 */
int mps_derive(const mps_params* p, mps_info* out);

/* ---- handle life cycle ------------------------------------------------------------ */

/* Make `device` current for the calling host thread; handles created afterwards on this
 * thread live on it (one process per GPU: call once per rank before mps_create). */
int mps_select_device(int32_t device);

/*
 * Create a solver for one scene. Replaces RdDat + AlcBkt + SetPara (kernel.cu:4-143,
 * 307-478): derives the lattice constants, allocates device state, uploads the
 * particles, builds the buckets and runs Surface_Edge (kernel.cu:1878-1879).
 * Particles outside the padded domain become GST (RdDat drops them, kernel.cu:117).
 */
int mps_create(const mps_params* p, int32_t n, const int8_t* typ, const void* pos,
               const void* vel, const void* nrm, mps_handle** out);

/*
 * Create one solver holding `nscenes` independent scenes that are advanced together.
 * counts[s] particles of scene s are stored consecutively in the arrays; ids are
 * global (scene s starts at sum(counts[0..s))). Every scene shares precision.
 */
int mps_create_batch(int32_t nscenes, const mps_params* p, const int32_t* counts,
                     const int8_t* typ, const void* pos, const void* vel, const void* nrm,
                     mps_handle** out);

int mps_destroy(mps_handle* h);
/* Queue the handle's work on `cuda_stream` (a cudaStream_t); NULL selects the handle's own
 * non-blocking stream, which is the default. With MPS_OPT_OVERLAP a step also uses a
 * second stream of the handle, forked from and joined back into this one, so work queued on
 * this stream after a step still runs after all of it. */
int mps_set_stream(mps_handle* h, void* cuda_stream);
int mps_set_option(mps_handle* h, int32_t option, int32_t value);
int mps_synchronize(mps_handle* h);

/*
 * Moving walls. The reference declares a rotating wall (`w`, `wallangle`, `rot_rad`,
 * class.cuh:117-121) and notes that Surface_Edge must run every step once walls move
 * (kernel.cu:1879), but moves none: its OBJ/OBJ2 particles are static walls. This call gives
 * every wall particle of `type` (MPS_OBJ or MPS_OBJ2) a prescribed rigid motion: rotation at
 * `omega` rad/s about the line through `center` along `axis`, and translation at
 * `velocity`; the centre moves with the walls. From the next mps_step on, each step ends by
 * moving those walls one time step (positions, inward normals and the wall velocity that
 * ChkCol uses, v + omega x r), rebuilding the wall buckets and rerunning Surface_Edge, so
 * that the next step's mirrors and collisions see them at the new time. Mirrors keep the
 * reference's zero velocity (kernel.cu:834-836). The motion accumulates in double from the
 * walls' place when it is set; omega = 0 and velocity = 0 stop it (the walls stay where they
 * are). mps_phase does not move walls. Single-scene handles only; the adjoint needs static
 * walls. axis may be NULL when omega is 0.
 */
int mps_set_wall_motion(mps_handle* h, int32_t type, const double center[3],
                        const double axis[3], double omega, const double velocity[3]);

/* ---- time stepping ---------------------------------------------------------------- */

/* Advance every scene by `nsteps` steps of the loop body kernel.cu:1904-1941. The end of a
 * step (the next step's first mirror generation and the bucket builds of the new positions)
 * is queued at the start of the next step, or before any call that reads the sorted state
 * (mps_phase, mps_get_mirrors of generation 0 or 1, mps_get_integrals, mps_autotune,
 * mps_adjoint_record); a state replaced with mps_set_state in between never builds it.
 * Results are the same either way. */
int mps_step(mps_handle* h, int32_t nsteps);
/* Run one method of the reference's step on its own (MPS_PHASE_*). */
int mps_phase(mps_handle* h, int32_t phase);

/* ---- state access (host buffers, id order; DevicetoHost, kernel.cu:1847-1869) ------- */

int mps_get_info(mps_handle* h, int32_t scene, mps_info* out);
/* Any pointer may be NULL. acc is the reference's d_Acc. */
int mps_get_state(mps_handle* h, int8_t* typ, void* pos, void* vel, void* acc, void* prs,
                  void* pav);
/* Replace the non-wall state (walls are static and ignored here). typ in {FLD, GST}. */
int mps_set_state(mps_handle* h, const int8_t* typ, const void* pos, const void* vel,
                  const void* acc, const void* prs, const void* pav);
/* WLLSE flags of every particle (Surface for non-walls), kernel.cu:553-668. */
int mps_get_wall_flags(mps_handle* h, int8_t* wllse);
/*
 * Mirror particles, sorted by slot id = i*MPS_NUM_MRR + k as in the reference's d_TypM
 * layout (kernel.cu:689-893). `which` = 2: the second generation of the last step (what the
 * reference's mirror arrays hold after a step: GenMRR at x*, read by PrsGrdTrm);
 * 1: the first generation (read by VscTrm, ChkCol, MkPrs). After mps_step, set 1 already
 * holds the next step's first generation, made from the new positions; after the
 * MPS_PHASE_* calls it is the set MkBkt_MRR produced last. 0: the raw (unculled) output of
 * the last GenMRR_nonslip phase. pos is SoA with stride `cap`; *n_out receives the count
 * even if it exceeds cap.
 */
int mps_get_mirrors(mps_handle* h, int32_t which, int32_t cap, int32_t* slot, void* pos,
                    void* prs, int32_t* n_out);
/* Per-particle diagnostic table [n_particles][MPS_DIAG_NCOL] and number density n_i. */
int mps_get_diag(mps_handle* h, int32_t* table, void* ndens);
int mps_get_counters(mps_handle* h, mps_counters* out);
/* Accumulated device time (ms) and launch count of kernel group `kernel` (MPS_K_*) over the
 * steps run with MPS_OPT_TIMING on; `reset` != 0 clears the accumulators afterwards. */
int mps_get_timing(mps_handle* h, int32_t kernel, double* total_ms, int64_t* launches,
                   int32_t reset);
/*
 * Autotuner (replaces the reference's fixed THREADS 512, const.cuh:48). Each candidate is
 * timed over `trial_steps` steps with CUDA events and the fastest kept, per kernel group:
 * VscTrm's candidates in flight (MPS_OPT_CANDIDATE_BATCH: 2, 4, 8), threads per block (128,
 * 64) and candidate source (MPS_OPT_STAGING); ChkCol/MkPrs, PrsGrdTrm and the mirror
 * generation with 128, 96, 64 or 32 threads per block; then ChkCol/MkPrs, PrsGrdTrm and
 * VscTrm at their alternate register bound (MPS_OPT_REGISTER_BOUND). The state is restored afterwards,
 * so tuning changes no result (no kernel's arithmetic depends on these shapes).
 * chosen[MPS_K_COUNT] receives the block sizes (may be NULL); mps_get_option reads the
 * other knobs. The choice is kept for the process: a handle created later with the same
 * precision, batched or not, and fluid count in the same power-of-two class starts from it.
 */
int mps_autotune(mps_handle* h, int32_t trial_steps, int32_t* chosen);
/* Current value of an option (MPS_OPT_BLOCK reads VscTrm's block size). */
int mps_get_option(mps_handle* h, int32_t opt, int32_t* value);
/*
 * Adjoint of a rollout. The reference has no derivative of its step; these two calls add
 * one behind the same state layout.
 *
 * mps_adjoint_record advances the handle `nsteps` steps (as mps_step) and keeps the state
 * every `checkpoint_every` steps on the device. Single-scene handles only.
 *
 * mps_adjoint_backward takes the adjoint of a scalar loss with respect to the final
 * positions and velocities (SoA x[n], y[n], z[n], doubles, particle-id order; NULL = zero)
 * and returns its gradients with respect to the positions and velocities at the start of
 * the rollout (same layout; NULL = not wanted) and to the kinematic viscosity knm_vsc
 * (*grad_nu, host memory; NULL = not wanted). Array pointers may be host or device
 * memory. Entries of wall particles are zero. It recomputes each segment from its
 * checkpoint, holding the recorded step's discrete choices fixed (neighbour lists, mirror
 * sets, collision branches, the pressure-minimum neighbour, clamps and deletions), and
 * leaves the handle at the final state of the rollout. It can be called again on the same
 * recording. MPS_ERR_OVERFLOW if a neighbour list of the rollout exceeded its capacity.
 * Device memory per step of one segment: two neighbour lists of 160 int32 per fluid
 * particle, about 200 bytes of state per fluid particle, and two mirror generations of
 * 10 slots x 68 bytes per fluid particle.
 */
int mps_adjoint_record(mps_handle* h, int32_t nsteps, int32_t checkpoint_every);
int mps_adjoint_backward(mps_handle* h, const double* lam_pos, const double* lam_vel,
                         double* grad_pos0, double* grad_vel0, double* grad_nu);
/*
 * Integrals of scene `scene`: out[0..2] fluid centroid, out[3] kinetic energy per unit
 * mass (sum |v|^2 / 2), out[4] surge front (max x of fluid), out[5] alive fluid count.
 */
int mps_get_integrals(mps_handle* h, int32_t scene, double out[6]);

/* ---- the reference's files (host only, no GPU needed) ------------------------------ */

/* MPS_physical.txt: 17 numbers in the order RdDat reads them (kernel.cu:12-22). */
typedef struct mps_physical {
    double min[3], max[3];   /* MIN, MAX: domain before the 3.1*l0 padding               */
    double g[3];             /* G [m/s^2]                                                */
    double fin_tim;          /* FIN_TIM: end time [s]                                    */
    double output_time;      /* output_time: interval between output files [s]           */
    double mach;             /* Mach number: SND = umax / Ma (kernel.cu:408)              */
    double courant;          /* CRT_NUM (read, unused by the step)                        */
    double col_rat;          /* COL_RAT                                                  */
    double dst_lmt_rat;      /* DST_LMT_RAT                                              */
    double knm_vsc;          /* KNM_VSC                                                  */
    double pcl_dst;          /* PCL_DST                                                  */
} mps_physical;

/* Read / write MPS_physical.txt. Every number is read as a float, as RdDat does. */
int mps_read_physical(const char* path, mps_physical* out);
int mps_write_physical(const char* path, const mps_physical* ph);
/*
 * Read initial.txt (RdDat, kernel.cu:59-131): a count, then one line
 * 'idx typ x y z nx ny nz g' per particle, read as floats. Particles outside the domain of
 * `ph` padded by 3.1*l0 are dropped (kernel.cu:121); walls, OBJ and OBJ2 store the negated
 * file normal, i.e. the inward normal (kernel.cu:126-128), other types a zero normal.
 * typ[cap], pos and nrm (double SoA) are filled in file order and packed to stride *n_out.
 * *n_out always receives the number kept; if it exceeds `cap`, or any output pointer is
 * NULL, MPS_ERR_ARG is returned and nothing else is defined (call again with cap >= *n_out).
 */
int mps_read_initial(const char* path, const mps_physical* ph, int32_t cap, int8_t* typ,
                     double* pos, double* nrm, int32_t* n_out);
/* Write initial.txt from id-ordered typ/pos/nrm (double SoA, stride n, inward normals). */
int mps_write_initial(const char* path, int32_t n, const int8_t* typ, const double* pos,
                      const double* nrm);
/*
 * SetPara's derived parameters (kernel.cu:396-415) from the physical file and the scene:
 * rho = 1000 (const.cuh:37), H = the fluid's extent along the axis of the largest |g|
 * component (the reference uses y), umax = sqrt(2|g|H), snd = umax / Ma, pmax = rho|g|H,
 * dt = l0 / (umax + snd). pos is double SoA with stride n.
 */
int mps_params_from_physical(const mps_physical* ph, int32_t n, const int8_t* typ,
                             const double* pos, int32_t precision, mps_params* out);

/* ---- output files (WrtDat / WrtDatWLL / WrtDat2, kernel.cu:161-304) ------------------ */

typedef struct mps_output mps_output;
/*
 * Open an output set in directory `dir` (which must exist) for handle `h`, and write the
 * wall files outputwall00000.csv and outputWLLvec00000.csv of the current state (WrtDatWLL).
 * The output object keeps device staging and pinned host buffers of the handle's size and
 * one writer thread. Close it before the handle is destroyed.
 */
int mps_output_open(mps_handle* h, const char* dir, mps_output** out);
/*
 * WrtDat: write output%05d.csv (fluid: position, velocity, speed, pressure, pav / opt_fqc)
 * and outputMRR%05d.csv (the second mirror generation, in slot order) for file number
 * `index`, then set pav = 0 on the device. `opt_fqc` is the number of steps summed into pav
 * since the last write (the reference's OPT_FQC). The state is copied on the device in the
 * handle's stream order; the call waits only until the GPU reaches that copy, and the files
 * are written by the writer thread while the caller queues further steps. One write is in
 * flight at a time: a second call first waits for the first's files. An I/O error of a
 * write is reported by the next call on the output object.
 */
int mps_output_write(mps_output* o, int32_t index, double opt_fqc);
/* WrtDat2: write seitei.txt (the fluid as a restart file, kernel.cu:251-276) of the
 * current state. */
int mps_output_restart(mps_output* o);
/* Wait for pending files, release the output object, return the first unreported error. */
int mps_output_close(mps_output* o);

/* ---- bucket build without allocation ---------------------------------------------- */

#define MPS_NOALLOC_MAX_ITEMS (1 << 20)   /* particles per call                         */
#define MPS_NOALLOC_MAX_BUCKETS (1 << 20) /* buckets of the scene's grid                 */

/*
 * MkBkt (kernel.cu:516-550) for callers that cannot allocate device memory, such as code
 * running inside another framework's memory pool, real-time loops that must not allocate
 * after start-up, or plug-ins handed only their input and output buffers. No counterpart in
 * the reference: it has no such entry point. Every temporary lives in one fixed array of
 * about 21 MB inside the library (held on every GPU that loads it, until exit), so nothing
 * is allocated per call; the caller passes device buffers:
 *   typ[n], pos (SoA x[n], y[n], z[n]; float, or double for MPS_F64) - inputs;
 *   cell[n]       bucket index ib of each particle, -1 for GST          - output;
 *   order[n]      ids of the non-GST particles sorted by (bucket, id); entries past
 *                 start[nbxyz] are left untouched                        - output;
 *   start[nbxyz+1] first position in `order` of every bucket             - output.
 * nbxyz is the grid size of `p` (mps_derive). Work is queued on `stream` (a cudaStream_t,
 * NULL = legacy default) and not synchronised. Sizes above MPS_NOALLOC_MAX_ITEMS particles
 * or MPS_NOALLOC_MAX_BUCKETS buckets are rejected with MPS_ERR_OVERFLOW. All calls on a
 * device share the array: calls whose work overlaps on the GPU race, so serialise them on
 * one stream. The first call on a device looks up the array's address there; make it
 * before any stream capture. That address is kept for the life of the process, so do not
 * call this entry point on a device after a cudaDeviceReset of it. A particle outside the
 * bucket grid gets the nearest edge bucket (its coordinates are clamped, as the solver
 * does) and nothing reports it: check positions first where particles may leave the domain.
 */
int mps_bucket_build_noalloc(const mps_params* p, int32_t n, const int8_t* typ, const void* pos,
                             int32_t* cell, int32_t* order, int32_t* start, void* stream);

/* ---- measurement ------------------------------------------------------------------ */
/* Work of the neighbour passes, counted on the device during the steps run with
 * MPS_OPT_DIAG (cumulative over the handle's life). The neighbour pairs themselves are the
 * columns of mps_get_diag. No counterpart in the reference. */
typedef struct mps_work {
    int64_t visc_candidates;  /* fluid candidates VscTrm's walk tested                   */
    int64_t list_candidates;  /* fluid candidates tested to build ChkCol/MkPrs's lists   */
    int64_t list_entries;     /* entries of those lists (read once by ChkCol/MkPrs, twice
                                 by PrsGrdTrm)                                           */
    int64_t reserved[5];
} mps_work;
int mps_get_work(mps_handle* h, mps_work* out);

/* Arithmetic throughput of the current device, measured by project-written micro-kernels
 * (eight independent chains per thread on every SM, CUDA events, best of three): the
 * denominators of the neighbour passes' compute roofline. A square root or division is
 * counted with the one dependent addition its chain needs. No counterpart in the
 * reference. */
typedef struct mps_arith {
    double fp32_fma_flops, fp64_fma_flops;    /* 2 flops per fused multiply-add       */
    double fp32_sqrt_per_s, fp32_div_per_s;   /* IEEE sqrt / division (round to nearest) */
    double fp64_sqrt_per_s, fp64_div_per_s;
    double warp_issue_per_s;                  /* 4 schedulers per SM at the rated clock */
    int32_t sms, clock_khz;
    double reserved[4];
} mps_arith;
int mps_measure_arith(mps_arith* out);

/* ---- errors ----------------------------------------------------------------------- */
const char* mps_status_string(int32_t status);
/* Text of the last failure on this thread (CUDA error string, argument check, ...). */
const char* mps_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* MPS_B200_H */
