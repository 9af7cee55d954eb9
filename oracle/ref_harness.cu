// ref_harness.cu -- drives the reference's own `class MPS` (TEST INFRASTRUCTURE ONLY).
//
// Compiled by ref_build.sh together with a build copy of the reference's kernel.cu. Every
// member of the reference's class is public (class.cuh:5-144), so the harness can do what
// RdDat does from files (kernel.cu:59-141) directly from arrays, then call the reference's
// own AlcBkt / SetPara / MkBkt / Surface_Edge / ... methods, and read the device arrays
// back. SetPara derives umax, SND, Pmax and dt from the fluid height along y and G.y
// (kernel.cu:399-415); the harness overwrites those scalars afterwards with the explicit
// values every other part of this project uses (they are passed by value at each launch).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "class.cuh"

struct RefParams {  // same field order as mps_params / oracle_params
    double pcl_dst, min[3], max[3], g[3], knm_vsc, col_rat, dst_lmt_rat, rho, snd, dt, umax, pmax;
    int32_t precision;
    int32_t reserved[7];
};

namespace {

template <class T> T* hmalloc(size_t n) { return static_cast<T*>(malloc(sizeof(T) * (n ? n : 1))); }

}  // namespace

extern "C" {

int ref_real_size() { return int(sizeof(real)); }

// pos/vel/nrm: SoA real arrays of n particles; nrm is the inward normal (WLLVec)
void* ref_create(const RefParams* p, int n, const int8_t* typ, const real* pos, const real* vel,
                 const real* nrm) {
    MPS* o = new MPS();
    // MPS_physical.txt values (kernel.cu:25-41)
    o->PCL_DST = real(p->pcl_dst);
    o->MINc.x = real(double(real(p->min[0])) - 3.1 * double(o->PCL_DST));
    o->MINc.y = real(double(real(p->min[1])) - 3.1 * double(o->PCL_DST));
    o->MINc.z = real(double(real(p->min[2])) - 3.1 * double(o->PCL_DST));
    o->MAXc.x = real(double(real(p->max[0])) + 3.1 * double(o->PCL_DST));
    o->MAXc.y = real(double(real(p->max[1])) + 3.1 * double(o->PCL_DST));
    o->MAXc.z = real(double(real(p->max[2])) + 3.1 * double(o->PCL_DST));
    o->G.x = real(p->g[0]);
    o->G.y = real(p->g[1]);
    o->G.z = real(p->g[2]);
    o->FIN_TIM = real(1);
    o->output_time = real(1);
    o->Ma = real(1);
    o->CRT_NUM = real(0.2);
    o->COL_RAT = real(p->col_rat);
    o->DST_LMT_RAT = real(p->dst_lmt_rat);
    o->KNM_VSC = real(p->knm_vsc);
    // initial.txt (kernel.cu:64-139); particles outside the padded box are dropped there,
    // callers pass none
    o->nP = n;
    o->Pos.x = hmalloc<real>(n); o->Pos.y = hmalloc<real>(n); o->Pos.z = hmalloc<real>(n);
    o->Vel.x = hmalloc<real>(n); o->Vel.y = hmalloc<real>(n); o->Vel.z = hmalloc<real>(n);
    o->Acc.x = hmalloc<real>(n); o->Acc.y = hmalloc<real>(n); o->Acc.z = hmalloc<real>(n);
    o->Prs = hmalloc<real>(n);
    o->pav = hmalloc<real>(n);
    o->Typ = hmalloc<char>(n);
    o->Dns = hmalloc<real>(Dns_Num);
    o->WLLVec.x = hmalloc<real>(n); o->WLLVec.y = hmalloc<real>(n); o->WLLVec.z = hmalloc<real>(n);
    o->WLLSE = hmalloc<char>(n);
    size_t nm = size_t(n) * NumMRR;
    o->PosM.x = hmalloc<real>(nm); o->PosM.y = hmalloc<real>(nm); o->PosM.z = hmalloc<real>(nm);
    o->VelM.x = hmalloc<real>(nm); o->VelM.y = hmalloc<real>(nm); o->VelM.z = hmalloc<real>(nm);
    o->PrsM = hmalloc<real>(nm);
    o->TypM = hmalloc<char>(nm);
    int nf = 0, nw = 0, nobj = 0;
    for (int i = 0; i < n; ++i) {
        o->Typ[i] = char(typ[i]);
        o->Pos.x[i] = pos[i]; o->Pos.y[i] = pos[n + i]; o->Pos.z[i] = pos[2 * size_t(n) + i];
        o->Vel.x[i] = vel[i]; o->Vel.y[i] = vel[n + i]; o->Vel.z[i] = vel[2 * size_t(n) + i];
        o->Acc.x[i] = o->Acc.y[i] = o->Acc.z[i] = real(0);
        o->Prs[i] = real(0);
        o->pav[i] = real(0);
        o->WLLVec.x[i] = nrm[i]; o->WLLVec.y[i] = nrm[n + i]; o->WLLVec.z[i] = nrm[2 * size_t(n) + i];
        if (typ[i] == FLD) { ++nf; o->WLLVec.x[i] = o->WLLVec.y[i] = o->WLLVec.z[i] = real(0); }
        if (typ[i] == WLL) ++nw;
        if (typ[i] == OBJ) ++nobj;
    }
    o->nPFLD = nf; o->nPWLL = nw; o->nPOBJ = nobj;
    o->AlcBkt();
    o->SetPara();
    // explicit parameters instead of SetPara's y-based derivation (kernel.cu:407-415)
    o->umax = real(p->umax);
    o->SND = real(p->snd);
    o->Prs_coef = o->SND * o->SND / o->n0_grad;
    o->Pmax = real(p->pmax);
    o->dt = real(p->dt);
    if (p->rho != 1000.0) {
        for (int k = 0; k < Dns_Num; ++k) o->Dns[k] = real(p->rho);
        cudaMemcpy(o->d_Dns, o->Dns, sizeof(real) * Dns_Num, cudaMemcpyHostToDevice);
    }
    // ClcMPS prologue (kernel.cu:1878-1879)
    o->MkBkt();
    o->Surface_Edge();
    if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
    return o;
}

// phase numbering = MPS_PHASE_* (include/mps_b200.h)
int ref_phase(void* h, int ph) {
    MPS* o = static_cast<MPS*>(h);
    switch (ph) {
        case 0: o->MkBkt(); break;
        case 1: o->Surface_Edge(); break;
        case 2: o->ResetMRR(); break;
        case 3: o->GenMRR_nonslip(); break;
        case 4: o->MkBkt_MRR(); break;
        case 5: o->VscTrm(); break;
        case 6: o->UpPcl1(); break;
        case 7: o->ChkCol(); break;
        case 8: o->MkPrs(); break;
        case 9: o->PrsGrdTrm(); break;
        case 10: o->UpPcl2(); break;
        default: return 1;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// one step = the loop body of ClcMPS (kernel.cu:1904-1935)
int ref_step(void* h, int nsteps) {
    MPS* o = static_cast<MPS*>(h);
    for (int s = 0; s < nsteps; ++s) {
        o->MkBkt();
        o->ResetMRR(); o->GenMRR_nonslip(); o->MkBkt_MRR();
        o->VscTrm();
        o->UpPcl1();
        o->MkBkt();
        o->ChkCol();
        o->MkBkt();
        o->MkPrs();
        o->ResetMRR(); o->GenMRR_nonslip(); o->MkBkt_MRR();
        o->PrsGrdTrm();
        o->UpPcl2();
        o->TIM += o->dt;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

int ref_get_state(void* h, int8_t* typ, real* pos, real* vel, real* acc, real* prs, real* pav) {
    MPS* o = static_cast<MPS*>(h);
    const int n = o->nP;
    o->DevicetoHost();
    std::vector<real> ax(n), ay(n), az(n);
    cudaMemcpy(ax.data(), o->d_Acc.x, sizeof(real) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(ay.data(), o->d_Acc.y, sizeof(real) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(az.data(), o->d_Acc.z, sizeof(real) * n, cudaMemcpyDeviceToHost);
    for (int i = 0; i < n; ++i) {
        typ[i] = int8_t(o->Typ[i]);
        pos[i] = o->Pos.x[i]; pos[n + i] = o->Pos.y[i]; pos[2 * size_t(n) + i] = o->Pos.z[i];
        vel[i] = o->Vel.x[i]; vel[n + i] = o->Vel.y[i]; vel[2 * size_t(n) + i] = o->Vel.z[i];
        acc[i] = ax[i]; acc[n + i] = ay[i]; acc[2 * size_t(n) + i] = az[i];
        prs[i] = o->Prs[i];
        pav[i] = o->pav[i];
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int ref_set_state(void* h, const int8_t* typ, const real* pos, const real* vel, const real* acc,
                  const real* prs, const real* pav) {
    MPS* o = static_cast<MPS*>(h);
    const int n = o->nP;
    std::vector<char> t(n);
    for (int i = 0; i < n; ++i) t[i] = char(typ[i]);
    cudaMemcpy(o->d_Typ, t.data(), n, cudaMemcpyHostToDevice);
    const real* src[] = {pos, pos + n, pos + 2 * size_t(n), vel, vel + n, vel + 2 * size_t(n),
                         acc, acc + n, acc + 2 * size_t(n)};
    real* dst[] = {o->d_Pos.x, o->d_Pos.y, o->d_Pos.z, o->d_Vel.x, o->d_Vel.y, o->d_Vel.z,
                   o->d_Acc.x, o->d_Acc.y, o->d_Acc.z};
    for (int k = 0; k < 9; ++k) cudaMemcpy(dst[k], src[k], sizeof(real) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(o->d_Prs, prs, sizeof(real) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(o->d_pav, pav, sizeof(real) * n, cudaMemcpyHostToDevice);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

int ref_get_wall_flags(void* h, int8_t* wse) {
    MPS* o = static_cast<MPS*>(h);
    std::vector<char> w(o->nP);
    cudaMemcpy(w.data(), o->d_WLLSE, o->nP, cudaMemcpyDeviceToHost);
    for (int i = 0; i < o->nP; ++i) wse[i] = int8_t(w[i]);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// mirror slots (reference layout, nP * NumMRR): type, position, pressure, source wall
int ref_get_mirrors(void* h, int8_t* typm, real* posm, real* prsm, int* fromwll) {
    MPS* o = static_cast<MPS*>(h);
    const size_t nm = size_t(o->nP) * NumMRR;
    std::vector<char> t(nm);
    cudaMemcpy(t.data(), o->d_TypM, nm, cudaMemcpyDeviceToHost);
    for (size_t k = 0; k < nm; ++k) typm[k] = int8_t(t[k]);
    cudaMemcpy(posm, o->d_PosM.x, sizeof(real) * nm, cudaMemcpyDeviceToHost);
    cudaMemcpy(posm + nm, o->d_PosM.y, sizeof(real) * nm, cudaMemcpyDeviceToHost);
    cudaMemcpy(posm + 2 * nm, o->d_PosM.z, sizeof(real) * nm, cudaMemcpyDeviceToHost);
    cudaMemcpy(prsm, o->d_PrsM, sizeof(real) * nm, cudaMemcpyDeviceToHost);
    if (fromwll) cudaMemcpy(fromwll, o->d_FromWLL, sizeof(int) * nm, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// bucket of every particle found by walking the reference's linked lists (bfst / nxt);
// -1 for particles in no list. Returns the number of list entries visited.
int ref_get_buckets(void* h, int* cell_of) {
    MPS* o = static_cast<MPS*>(h);
    const int n = o->nP, nb = o->nBxyz;
    std::vector<int> bfst(nb), nxt(n);
    cudaMemcpy(bfst.data(), o->d_bfst, sizeof(int) * nb, cudaMemcpyDeviceToHost);
    cudaMemcpy(nxt.data(), o->d_nxt, sizeof(int) * n, cudaMemcpyDeviceToHost);
    for (int i = 0; i < n; ++i) cell_of[i] = -1;
    int visited = 0;
    for (int b = 0; b < nb; ++b) {
        int j = bfst[b];
        int guard = 0;
        while (j >= 0 && j < n && guard++ <= n) {
            cell_of[j] = b;
            ++visited;
            j = nxt[j];
        }
    }
    return visited;
}

// the particles of every bucket in the order of the reference's linked lists (bfst / nxt):
// order[start[b] .. start[b+1]) for bucket b; start has nBxyz + 1 entries. Returns the number
// of entries written (at most cap).
int ref_get_list_order(void* h, int cap, int* order, int* start) {
    MPS* o = static_cast<MPS*>(h);
    const int n = o->nP, nb = o->nBxyz;
    std::vector<int> bfst(nb), nxt(n);
    cudaMemcpy(bfst.data(), o->d_bfst, sizeof(int) * nb, cudaMemcpyDeviceToHost);
    cudaMemcpy(nxt.data(), o->d_nxt, sizeof(int) * n, cudaMemcpyDeviceToHost);
    int at = 0;
    for (int b = 0; b < nb; ++b) {
        start[b] = at;
        int j = bfst[b], guard = 0;
        while (j >= 0 && j < n && guard++ <= n) {
            if (at < cap) order[at] = j;
            ++at;
            j = nxt[j];
        }
    }
    start[nb] = at;
    return at;
}

// derived constants: n0, lmd, n0_grad, lmd_grad, Numn0_grad, r, rp, DB, DBinv, nBx, nBy, nBz,
// rlim2, COL, Prs_coef, MINc xyz, MAXc xyz
int ref_get_info(void* h, double* out) {
    MPS* o = static_cast<MPS*>(h);
    double v[] = {double(o->n0), double(o->lmd), double(o->n0_grad), double(o->lmd_grad),
                  double(o->Numn0_grad), double(o->r), double(o->rp), double(o->DB),
                  double(o->DBinv), double(o->nBx), double(o->nBy), double(o->nBz),
                  double(o->rlim2), double(o->COL), double(o->Prs_coef), double(o->MINc.x),
                  double(o->MINc.y), double(o->MINc.z), double(o->MAXc.x), double(o->MAXc.y),
                  double(o->MAXc.z)};
    memcpy(out, v, sizeof(v));
    return 0;
}

}  // extern "C"
