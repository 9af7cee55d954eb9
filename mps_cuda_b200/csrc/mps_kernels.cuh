// mps_kernels.cuh -- sm_100a kernels of the explicit MPS step.
//
// Bucket build (replaces d_MkBkt's atomicExch linked list, kernel.cu:516-550):
//   key   : bucket of every item, warp-aggregated atomicAdd on the bucket counter
//   scan  : exclusive scan of the counters -> bucket start table (two launches)
//   seg   : scatter ids into their bucket segment (arbitrary order inside a bucket)
//   fin   : rank every item by id inside its bucket and gather its payload to the new slot
// The result is deterministic: bucket-major, ascending id inside a bucket.
//
// Fused step (kernel.cu:1904-1935 in three neighbour passes):
//   pass A: VscTrm + UpPcl1 (+ChkPcl)                            reads x^n, v^n, M1
//   pass B: ChkCol + MkPrs + GenMRR/MRRinout at (x*, P)          reads x*, v*, walls, M1
//   pass C: PrsGrdTrm + UpPcl2 (+ChkPcl) + GenMRR/MRRinout at (x^{n+1}, P)  reads x*, P, M2
// Mirrors produced by pass C are the next step's first generation: GenMRR at the start of
// the next step (kernel.cu:1906-1908) would read the same positions and pressures.
#pragma once
#include <climits>
#include <type_traits>

#include "mps_device.cuh"

namespace mps {

constexpr int kDiagCols = 11;
enum { DG_CELL = 0, DG_VSC_F, DG_VSC_M, DG_COL_F, DG_COL_W, DG_COL_M, DG_PRS_F, DG_PRS_M,
       DG_GRD_F, DG_GRD_M, DG_GEN_W };

// ---------------------------------------------------------------------------------------
// bucket build
// ---------------------------------------------------------------------------------------
template <class R, class RN> struct FluidKeySrc {
    const SceneDev<R, RN>* sc;
    int nscene, dead;
    const V4<R>* pos;
    const int8_t* typ;
    const int* pid;
    __device__ __forceinline__ int key(int t, DevCounters* cnt) const {
        if (typ[t] != kFLD) return dead;
        int id = pid[t];
        int s = nscene > 1 ? scene_of(sc, nscene, id) : 0;
        V4<R> p = pos[t];
        if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) atomicAdd(&cnt->err_nan, 1);
        bool ok;
        const int c = fine_cell(sc[s], p.x, p.y, p.z, ok);
        if (!ok) atomicAdd(&cnt->err_cell, 1);
        return c;
    }
    __device__ __forceinline__ int id(int t) const { return pid[t]; }
};

template <class R, class RN> struct WallKeySrc {
    const SceneDev<R, RN>* sc;
    int nscene, dead;
    const V4<R>* pos;
    const int* wid;
    __device__ __forceinline__ int key(int t, DevCounters* cnt) const {
        int id = wid[t];
        int s = nscene > 1 ? scene_of(sc, nscene, id) : 0;
        V4<R> p = pos[t];
        int ix, iy, iz;
        if (!cell_of(sc[s], p.x, p.y, p.z, ix, iy, iz)) atomicAdd(&cnt->err_cell, 1);
        return sc[s].cbase + iz * sc[s].nbxy + iy * sc[s].nbx + ix;
    }
    __device__ __forceinline__ int id(int t) const { return wid[t]; }
};

template <class R, class RN> struct MirrorKeySrc {
    const SceneDev<R, RN>* sc;
    int nscene, dead;
    const V4<R>* pos;
    const int* slot;
    __device__ __forceinline__ int key(int t, DevCounters* cnt) const {
        int sl = slot[t];
        if (sl < 0) return dead;  // culled
        int s = nscene > 1 ? scene_of(sc, nscene, sl / kNumMRR) : 0;
        V4<R> p = pos[t];
        int ix, iy, iz;
        if (!cell_of(sc[s], p.x, p.y, p.z, ix, iy, iz)) atomicAdd(&cnt->err_cell, 1);
        return sc[s].cbase + iz * sc[s].nbxy + iy * sc[s].nbx + ix;
    }
    __device__ __forceinline__ int id(int t) const { return slot[t]; }
};

__device__ __forceinline__ int item_count(const int* n_ptr, int n_fixed) {
    return n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
}

constexpr int kScan16Threads = 512, kScan16Per = 16, kScan16Tile = kScan16Threads * kScan16Per;

// Adds each lane's item to part[tile] (tile < 0: no item), one atomic per run of lanes with
// the same tile: items arrive nearly sorted by bucket (a warp's mirrors come from
// neighbouring particles), so a warp's tiles form a few runs. Every lane of the warp calls
// this.
__device__ __forceinline__ void tile_runs_add(int tile, int lane, int* __restrict__ part) {
    const int prev = __shfl_up_sync(0xffffffffu, tile, 1);
    const bool start = lane == 0 || tile != prev;
    const unsigned starts = __ballot_sync(0xffffffffu, start);
    if (start && tile >= 0) {
        const unsigned later = starts & ~((2u << lane) - 1u);
        const int end = later ? __ffs(later) - 1 : 32;
        atomicAdd(&part[tile], end - lane);
    }
}

template <class Src>
__global__ void k_bin_key(Src src, const int* n_ptr, int n_fixed, int* __restrict__ key,
                          int* __restrict__ rnk, int* __restrict__ count, int* __restrict__ part,
                          DevCounters* cnt) {
    // part (may be null): per kScan16Tile tile totals of count, for k_fine_scan
    const int n = item_count(n_ptr, n_fixed);
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    // whole warps iterate together so that the warp-aggregated atomic sees every lane
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        int t = base + lane;
        bool act = t < n;
        int c = act ? src.key(t, cnt) : -1;
        unsigned peers = __match_any_sync(0xffffffffu, c);
        int leader = __ffs(peers) - 1;
        int below = __popc(peers & ((1u << lane) - 1));
        int b = 0;
        if (act && lane == leader) b = atomicAdd(&count[c], __popc(peers));
        if (part) tile_runs_add(act ? c / kScan16Tile : -1, lane, part);  // uniform branch
        b = __shfl_sync(0xffffffffu, b, leader);
        if (act) {
            key[t] = c;
            rnk[t] = b + below;
        }
    }
}


template <class Src>
__global__ void k_bin_seg(Src src, const int* n_ptr, int n_fixed, const int* __restrict__ key,
                          const int* __restrict__ rnk, const int* __restrict__ cs,
                          int* __restrict__ seg) {
    const int n = item_count(n_ptr, n_fixed);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        seg[cs[key[t]] + rnk[t]] = src.id(t);
}

template <class Src, class G>
__global__ void k_bin_fin(Src src, G g, const int* n_ptr, int n_fixed, const int* __restrict__ key,
                          const int* __restrict__ rnk, const int* __restrict__ cs,
                          const int* __restrict__ seg, int dead) {
    const int n = item_count(n_ptr, n_fixed);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        int c = key[t];
        int lo = __ldg(cs + c);
        int d;
        if (c == dead) {
            d = lo + rnk[t];  // order of unlisted items is irrelevant
        } else {
            int hi = __ldg(cs + c + 1), my = src.id(t), r = 0;
            for (int k = lo; k < hi; ++k) r += (__ldg(seg + k) < my);
            d = lo + r;
        }
        g(t, d);
    }
}

template <class R> struct FluidGather {
    const V4<R>* pos; const V4<R>* vel; const V4<R>* acc;
    const R* prs; const R* pav; const int* pid; const int8_t* typ;
    V4<R>* dpos; V4<R>* dvel; V4<R>* dacc;
    R* dprs; R* dpav; int* dpid; int8_t* dtyp;
    __device__ __forceinline__ void operator()(int t, int d) const {
        int8_t ty = typ[t];
        dpos[d] = pos[t];
        dvel[d] = vel[t];
        if (acc) dacc[d] = acc[t];
        dprs[d] = ty == kFLD ? prs[t] : R(0);
        dpav[d] = pav[t];
        dpid[d] = pid[t];
        dtyp[d] = ty;
    }
};

template <class R> struct MirrorGather {
    const V4<R>* pos; const int* slot;
    V4<R>* dpos; int* dslot;
    __device__ __forceinline__ void operator()(int t, int d) const {
        dpos[d] = pos[t];
        dslot[d] = slot[t];
    }
};

// FluidGather that also writes the row-ordered position copy: an item of fine cell c
// (bucket-major, starts cs) that lands in slot d goes to posf[csr[rowmajor(c)] + d - cs[c]]
// with its slot in w. Inside a fine cell both orders are ascending id.
template <class R, class RN> struct FluidGatherF {
    FluidGather<R> g;
    const SceneDev<R, RN>* sc;
    int nscene;
    const int* key; const int* cs; const int* csr;
    V4<R>* posf;
    __device__ __forceinline__ void operator()(int t, int d) const {
        g(t, d);
        if (g.typ[t] != kFLD) return;
        const int c = key[t];
        const int id = g.pid[t];
        const SceneDev<R, RN>& s = sc[nscene > 1 ? scene_of(sc, nscene, id) : 0];
        const V4<R> p = g.pos[t];
        posf[__ldg(csr + fine_rowmajor(s, c)) + d - __ldg(cs + c)] = V4<R>{p.x, p.y, p.z, slot_w(d, R(0))};
    }
};

// positions of the row-ordered copy from the slots' current positions (the per-method
// path moves particles in place between bucket builds)
template <class R>
__global__ void k_posf_refresh(V4<R>* posf, const V4<R>* __restrict__ pos, const int* __restrict__ csr,
                               int ncell) {
    const int n = __ldg(csr + ncell);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const V4<R> q = posf[k];
        const V4<R> p = pos[w_slot(q.w)];
        posf[k] = V4<R>{p.x, p.y, p.z, q.w};
    }
}

// MirrorGather that also carries the recorded reflection normals
template <class R> struct MirrorGatherN {
    const V4<R>* pos; const int* slot; const V4<R>* nrm;
    V4<R>* dpos; int* dslot; V4<R>* dnrm;
    __device__ __forceinline__ void operator()(int t, int d) const {
        dpos[d] = pos[t];
        dslot[d] = slot[t];
        dnrm[d] = nrm[t];
    }
};

template <class R> struct WallGather {
    const V4<R>* pos; const V4<R>* nrm; const V4<R>* vel; const int* wid; const int8_t* typ;
    V4<R>* dpos; V4<R>* dnrm; V4<R>* dvel; int* dwid; int8_t* dtyp;
    __device__ __forceinline__ void operator()(int t, int d) const {
        dpos[d] = pos[t];
        dnrm[d] = nrm[t];
        dvel[d] = vel[t];
        dwid[d] = wid[t];
        dtyp[d] = typ[t];
    }
};

// exclusive scan of count[0..L) into out[0..L], out[L] = total
constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ int block_sum(int v, int* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    int t = 0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    int r = sh[0];
    __syncthreads();
    return r;
}

static __global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int* __restrict__ in, int L,
                                                              int* __restrict__ part) {
    __shared__ int sh[32];
    int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
    int v = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) v += (base + k < L) ? in[base + k] : 0;
    int s = block_sum(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

static __global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int* __restrict__ in, int L,
                                                             const int* __restrict__ part,
                                                             int* __restrict__ out) {
    __shared__ int sh[32];
    __shared__ int wsum[32];
    // offset of this tile = sum of the partials before it
    int off = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) off += part[b];
    off = block_sum(off, sh);
    int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
    int v[kScanPer], loc = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = (base + k < L) ? in[base + k] : 0;
        loc += v[k];
    }
    // inclusive warp scan of the thread sums
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = loc;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        int ws = lane < (blockDim.x >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        wsum[lane] = ws;  // inclusive over warps
    }
    __syncthreads();
    int excl = off + (w > 0 ? wsum[w - 1] : 0) + inc - loc;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (base + k < L) out[base + k] = excl;
        excl += v[k];
    }
    if (base <= L - 1 && L - 1 < base + kScanPer) out[L] = excl;  // thread holding the last item
}

// Scan of a bucket build's counts (k_fine_scan below): 16 counts per thread through int4
// loads, and the counts cleared as they are read, so that the next bucket build starts from
// zeros without a memset.

__device__ __forceinline__ void load16(const int* __restrict__ in, int base, int L, int v[16]) {
    if (base + 16 <= L) {
        const int4* p = reinterpret_cast<const int4*>(in + base);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int4 a = p[q];
            v[4 * q] = a.x; v[4 * q + 1] = a.y; v[4 * q + 2] = a.z; v[4 * q + 3] = a.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = (base + k < L) ? in[base + k] : 0;
    }
}

// Count tables of a bucket build with their per-tile totals (from the key kernel): the wall
// and mirror builds' bucket tables (gridDim.y = 1), count[k] scanned into out[k].
struct FineScan {
    int* count[2];
    int* part[2];
    int* out[2];
    int L, ntile;
    int* ticket;  // blocks finished; zero between launches
};

// Exclusive scan of count[k][0..L) into out[k][0..L], out[k][L] = total, for k = blockIdx.y.
// The counts are left zero; the last block to finish also zeroes the tile totals for the
// next build (every block has read them by then), so a build needs no memset.
static __global__ void __launch_bounds__(kScan16Threads) k_fine_scan(FineScan f) {
    __shared__ int sh[32];
    __shared__ int wsum[32];
    __shared__ int last;
    const int which = blockIdx.y, L = f.L;
    int* __restrict__ in = f.count[which];
    const int* __restrict__ part = f.part[which];
    int* __restrict__ out = f.out[which];
    int off = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) off += part[b];
    off = block_sum(off, sh);
    const int base = blockIdx.x * kScan16Tile + threadIdx.x * kScan16Per;
    int v[16];
    load16(in, base, L, v);
    int loc = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) loc += v[k];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = loc;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        int ws = lane < (blockDim.x >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        wsum[lane] = ws;
    }
    __syncthreads();
    int e[16];
    int excl = off + (w > 0 ? wsum[w - 1] : 0) + inc - loc;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        e[k] = excl;
        excl += v[k];
    }
    if (base + 16 <= L) {
        int4* o4 = reinterpret_cast<int4*>(out + base);
        int4* i4 = reinterpret_cast<int4*>(in + base);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            o4[q] = make_int4(e[4 * q], e[4 * q + 1], e[4 * q + 2], e[4 * q + 3]);
            i4[q] = make_int4(0, 0, 0, 0);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 16; ++k)
            if (base + k < L) {
                out[base + k] = e[k];
                in[base + k] = 0;
            }
    }
    if (base <= L - 1 && L - 1 < base + kScan16Per) out[L] = excl;  // thread holding the last item
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(f.ticket, 1) == int(gridDim.x * gridDim.y) - 1;
    }
    __syncthreads();
    if (last) {
        for (int k = threadIdx.x; k < f.ntile; k += blockDim.x)
            for (int y = 0; y < int(gridDim.y); ++y) f.part[y][k] = 0;
        if (threadIdx.x == 0) *f.ticket = 0;
    }
}

// ---------------------------------------------------------------------------------------
// start tables of the fluid build from one count table, by bucket rows
// ---------------------------------------------------------------------------------------
// The fluid's fine cells are counted once, bucket-major (27 per bucket, 9 sz + 3 sy + sx).
// A bucket row (one scene's buckets at iz, iy, every ix) holds 27 nbx of them: nine fine
// rows (3 iz + sz, 3 iy + sy) of 3 nbx cells each, interleaved bucket by bucket. Both start
// tables follow from per-row totals: the bucket-major one (cs) from each bucket row's total,
// the row-major one (csr, the order of posf) from each fine row's total. One block per
// bucket row totals its counts (k_fine_rows_sum), one block per table scans the totals
// (k_fine_rows_scan), and one block per bucket row writes both tables and clears its counts
// (k_fine_rows_write): the counts are read twice and cleared once, with no second count
// table and no second count atomic per item. (Taking the row totals in the key kernel
// instead, with one atomic per group of a warp's items in a row, was measured slower: the
// write pass then met the counts cold in DRAM.)
struct FineRows {
    int* count;          // bucket-major fine-cell counts (cleared by k_fine_rows_write)
    int* brtot;          // per bucket row (scene, iz, iy): its total, then its start
    int* frtot;          // per fine row (scene, fz, fy): its total, then its start
    int* cs;             // bucket-major starts, [0, dead + 1]
    int* csr;            // row-major starts, [0, dead + 1]
    const int* rowscan;  // per scene: bucket rows before it (nscene + 1 entries)
    int nscene, nrows;   // bucket rows of all scenes
    int dead;            // the unlisted items' cell, after every scene's cells
};

template <class R, class RN>
__device__ __forceinline__ const SceneDev<R, RN>& bucket_row(const FineRows& f,
                                                             const SceneDev<R, RN>* scs, int r,
                                                             int& s, int& iz, int& iy) {
    int lo = 0, hi = f.nscene;  // rowscan[lo] <= r < rowscan[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(f.rowscan + mid) <= r) lo = mid; else hi = mid;
    }
    s = lo;
    const SceneDev<R, RN>& sc = scs[s];
    const int lr = r - __ldg(f.rowscan + s);
    iz = lr / sc.nby;
    iy = lr - iz * sc.nby;
    return sc;
}

// fine row index (scene base + fz 3 nby + fy) of fine row q = 3 sz + sy of bucket row (iz, iy)
template <class R, class RN>
__device__ __forceinline__ int fine_row_of(const FineRows& f, const SceneDev<R, RN>& sc, int s,
                                           int iz, int iy, int q) {
    return 9 * __ldg(f.rowscan + s) + (3 * iz + q / 3) * (3 * sc.nby) + 3 * iy + q % 3;
}

// inclusive warp scan of v (all lanes)
__device__ __forceinline__ int warp_incl(int v) {
    const int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// exclusive block scan of the N values of every thread; tot receives the block totals.
// sh: N * 32 ints of shared memory
template <int N>
__device__ __forceinline__ void block_exscan(int (&v)[N], int (&tot)[N], int* sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int inc[N];
#pragma unroll
    for (int q = 0; q < N; ++q) inc[q] = warp_incl(v[q]);
    __syncthreads();
    if (lane == 31)
#pragma unroll
        for (int q = 0; q < N; ++q) sh[q * 32 + w] = inc[q];
    __syncthreads();
    if (w == 0)
#pragma unroll
        for (int q = 0; q < N; ++q) {
            const int x = lane < nw ? sh[q * 32 + lane] : 0;
            sh[q * 32 + lane] = warp_incl(x);  // inclusive over warps
        }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < N; ++q) {
        const int before = w > 0 ? sh[q * 32 + w - 1] : 0;
        tot[q] = sh[q * 32 + nw - 1];
        v[q] = before + inc[q] - v[q];
    }
    __syncthreads();
}

// A chunk of T buckets of a bucket row (T threads per block: 64, 128 or 256, the handle's
// longest bucket row rounded up, so that short rows do not leave most threads idle) moves
// between global and shared memory with coalesced loads and stores; each thread then works on
// its own bucket's 27 counts there (stride 27, odd: no bank conflicts).

template <class R, class RN, int T>
__global__ void __launch_bounds__(T) k_fine_rows_sum(FineRows f,
                                                                const SceneDev<R, RN>* scs) {
    __shared__ int sh[9 * 32];
    __shared__ int buf[27 * T];
    int s, iz, iy;
    const SceneDev<R, RN>& sc = bucket_row(f, scs, blockIdx.x, s, iz, iy);
    const int* __restrict__ cnt = f.count + sc.fbase + 27 * (iz * sc.nbxy + iy * sc.nbx);
    int t9[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) t9[q] = 0;
    for (int b0 = 0; b0 < sc.nbx; b0 += T) {
        const int n = 27 * min(T, sc.nbx - b0);
        __syncthreads();
        // unrolled with a fixed trip count, so that a thread's 27 loads are in flight together
#pragma unroll
        for (int j = 0; j < 27; ++j) {
            const int i = threadIdx.x + j * T;
            if (i < n) buf[i] = __ldg(cnt + 27 * b0 + i);
        }
        __syncthreads();
        if (27 * threadIdx.x < n)
#pragma unroll
            for (int k = 0; k < 27; ++k) t9[k / 3] += buf[27 * threadIdx.x + k];
    }
    int tot[9];
    block_exscan<9>(t9, tot, sh);
    if (threadIdx.x == 0) {
        int all = 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            f.frtot[fine_row_of(f, sc, s, iz, iy, q)] = tot[q];
            all += tot[q];
        }
        f.brtot[blockIdx.x] = all;
    }
}

// exclusive scan in place of brtot (block 0, nrows entries) and frtot (block 1, 9 nrows);
// block 0 also closes both tables with the unlisted cell and clears its count. Each warp
// scans one contiguous segment 32 entries at a time (coalesced), after one pass that totals
// the segments.
static __global__ void __launch_bounds__(1024) k_fine_rows_scan(FineRows f) {
    __shared__ int sh[32];
    int* a = blockIdx.x == 0 ? f.brtot : f.frtot;
    const int n = blockIdx.x == 0 ? f.nrows : 9 * f.nrows;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int seg = (n + nw - 1) / nw;
    const int lo = min(n, w * seg), hi = min(n, lo + seg);
    int sum = 0;
#pragma unroll 4
    for (int k = lo + lane; k < hi; k += 32) sum += a[k];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) sh[w] = sum;
    __syncthreads();
    if (w == 0) {
        const int x = lane < nw ? sh[lane] : 0;
        const int inc = warp_incl(x);
        __syncwarp();
        sh[lane] = inc - x;  // exclusive start of each warp's segment
        if (blockIdx.x == 0 && lane == 31) {
            const int total = inc;  // every listed item
            const int nd = f.count[f.dead];
            f.cs[f.dead] = total;
            f.cs[f.dead + 1] = total + nd;
            f.csr[f.dead] = total;
            f.csr[f.dead + 1] = total + nd;
            f.count[f.dead] = 0;
        }
    }
    __syncthreads();
    int run = sh[w];
    for (int k0 = lo; k0 < hi; k0 += 128) {  // four loads in flight per lane
        int x[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = k0 + 32 * j + lane;
            x[j] = k < hi ? a[k] : 0;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = k0 + 32 * j + lane;
            const int inc = warp_incl(x[j]);
            if (k < hi) a[k] = run + inc - x[j];
            run += __shfl_sync(0xffffffffu, inc, 31);
        }
    }
}

template <class R, class RN, int T>
__global__ void __launch_bounds__(T) k_fine_rows_write(FineRows f,
                                                                  const SceneDev<R, RN>* scs) {
    __shared__ int sh[10 * 32];
    __shared__ int carry[10];  // bucket-major, then the nine fine rows
    __shared__ int buf[27 * T];
    int s, iz, iy;
    const SceneDev<R, RN>& sc = bucket_row(f, scs, blockIdx.x, s, iz, iy);
    const int cb = sc.fbase + 27 * (iz * sc.nbxy + iy * sc.nbx);
    int* __restrict__ cnt = f.count + cb;
    if (threadIdx.x < 10)
        carry[threadIdx.x] = threadIdx.x == 0
                                 ? __ldg(f.brtot + blockIdx.x)
                                 : __ldg(f.frtot + fine_row_of(f, sc, s, iz, iy, threadIdx.x - 1));
    const int nfx = 3 * sc.nbx, nfxy = 9 * sc.nbxy;
    for (int b0 = 0; b0 < sc.nbx; b0 += T) {
        const int nb = min(T, sc.nbx - b0), n = 27 * nb;
        const bool act = int(threadIdx.x) < nb;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 27; ++j) {
            const int i = threadIdx.x + j * T;
            if (i < n) buf[i] = cnt[27 * b0 + i];
        }
        __syncthreads();
        int c[27];
#pragma unroll
        for (int k = 0; k < 27; ++k) c[k] = act ? buf[27 * threadIdx.x + k] : 0;
        int v[10], tot[10];
        v[0] = 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            v[q + 1] = c[3 * q] + c[3 * q + 1] + c[3 * q + 2];
            v[0] += v[q + 1];
        }
        block_exscan<10>(v, tot, sh);  // also orders the reads of buf before the writes below
        // bucket-major starts, through buf
        if (act) {
            int run = carry[0] + v[0];
#pragma unroll
            for (int k = 0; k < 27; ++k) {
                buf[27 * threadIdx.x + k] = run;
                run += c[k];
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 27; ++j) {
            const int i = threadIdx.x + j * T;
            if (i < n) {
                f.cs[cb + 27 * b0 + i] = buf[i];
                cnt[27 * b0 + i] = 0;  // the counts back to zero for the next build
            }
        }
        // row-major starts: fine row q's 3 nb cells of this chunk are contiguous in csr
        __syncthreads();
        if (act)
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                int r = carry[q + 1] + v[q + 1];
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    buf[q * 3 * T + 3 * threadIdx.x + x] = r;
                    r += c[3 * q + x];
                }
            }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            int* o = f.csr + sc.fbase + (3 * iz + q / 3) * nfxy + (3 * iy + q % 3) * nfx + 3 * b0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int i = threadIdx.x + j * T;
                if (i < 3 * nb) o[i] = buf[q * 3 * T + i];
            }
        }
        if (threadIdx.x < 10) carry[threadIdx.x] += tot[threadIdx.x];
    }
}

// ---------------------------------------------------------------------------------------
// neighbour passes
// ---------------------------------------------------------------------------------------
// Entry k of slot s's neighbour list. The 32 slots of a warp own one contiguous tile of
// K x 32 entries, entry-major (a warp's entry k is one 128-byte line). A layout strided by the
// slot count instead spreads a warp's lines over the whole list, so that each line leaves L2
// between its lanes' partial writes and is written back several times (measured: about three
// times the list's bytes in DRAM writes at 2.9M particles).
__device__ __forceinline__ size_t list_at(int s, int k, int K) {
    return (size_t(s >> 5) * size_t(K) + size_t(k)) * 32 + size_t(s & 31);
}

// Resident blocks per SM asked of a kernel tuned in FP32: half as many in FP64, whose values
// take two registers each (at the FP32 bound the FP64 kernels spill).
template <class R> constexpr int min_blocks(int f32) { return sizeof(R) == 8 ? f32 / 2 : f32; }

// Two register bounds each for passes A, B and C (MPS_OPT_REGISTER_BOUND, chosen by the
// autotuner); which is faster depends on the grid's size, the precision and pass A's
// candidate batch. Passes A and B: 8 resident blocks of 128 threads per SM in FP32 (64
// registers) and 5 in FP64 (up to 102), or one block more (FP32 56 registers, FP64 80) with
// a few spills. Pass C: 8 blocks per SM (FP32 64 registers without spills, FP64 64 with
// about 200 bytes of spills), or FP32 10 blocks (48) and FP64 4 blocks (122, no spills).
// Measured with CUDA events at 6.1M particles in FP32, the alternate bounds take pass A
// from 3.77 to 3.72 ms, pass B from 2.34 to 2.09 ms and pass C from 1.18 to 1.11 ms; in FP64
// the spill-free pass C is 9 % faster at 48 000 particles and 10 % slower at 384 000.
template <class R> constexpr int pass_a_blocks(bool alt) {
    return sizeof(R) == 8 ? (alt ? 6 : 5) : (alt ? 9 : 8);
}
template <class R> constexpr int pass_b_blocks(bool alt) {
    return sizeof(R) == 8 ? (alt ? 6 : 5) : (alt ? 9 : 8);
}
template <class R> constexpr int pass_c_blocks(bool alt, bool corr) {
    return corr ? min_blocks<R>(6) : alt ? (sizeof(R) == 8 ? 4 : 10) : 8;
}

// The step kernels take this as a `const __grid_constant__` parameter. The out-of-line walks
// receive references to its views (wl, m); an ordinary by-value kernel parameter whose address
// is taken is copied whole into local memory by every thread (measured: a 376-byte stack frame
// in pass C and 480 in pass B, about 11 and 30 sectors of local stores per particle).
template <class R, class RN> struct PassArgs {
    const SceneDev<R, RN>* sc;
    int nscene, nF, dead, skip;
    const int* cs;  // fluid bucket starts
    // sorted state
    V4<R>* pos; V4<R>* vel; V4<R>* acc; R* prs; R* pav; const int* pid; int8_t* typ;
    // scratch in the same slot order
    V4<R>* tpos; V4<R>* tvel; R* tprs; int8_t* ttyp;
    WallView<R> wl;
    MirrorView<R> m;
    MirrorSink<R> out;
    DevCounters* cnt;
    int32_t* diag;
    RN* ndens;
    // neighbour lists: entry k of slot s (its k-th neighbour in visiting order) is
    // nb[list_at(s, k, nbK)]; nbcnt[s] is the list's length (lists longer than nbK fall back
    // to a scan)
    int* nb;
    int* nbcnt;
    int nbK;
    const int8_t* near_wall;  // per bucket: a wall lies in the 27 buckets around it
    // per bucket: a mirror of the view `m` lies in the 27 buckets around it (null: walk
    // the mirrors everywhere). The wall and mirror walks visit only a particle's 27 buckets,
    // so skipping them where these flags are clear changes no sum.
    const int8_t* near_m;
    // recorded rollouts only: per slot the velocity before ChkPcl's clamp, w = slot state
    // (kTapeOk, kTapeClamped, kTapeDeleted, kTapeDead)
    V4<R>* tape_pre;
    // fluid positions in row-major fine-cell order, w = slot; csr its fine-cell starts
    const V4<R>* posf;
    const int* csr;
};

// near flag of every bucket of every scene: some item of the bucket table `wcs` (walls, or
// the mirrors of one generation) lies in the 27 buckets around it
template <class R, class RN>
__global__ void k_near_wall(const SceneDev<R, RN>* scs, int nscene, const int* __restrict__ wcs,
                            int8_t* near_wall) {
    const int sidx = blockIdx.y;
    const SceneDev<R, RN>& sc = scs[sidx];
    const int nb = sc.nbxy * sc.nbz;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int iz = b / sc.nbxy, iy = (b % sc.nbxy) / sc.nbx, ix = b % sc.nbx;
        int8_t f = 1;  // buckets on the grid border hold no particle: keep them conservative
        if (ix >= 1 && ix <= sc.nbx - 2 && iy >= 1 && iy <= sc.nby - 2 && iz >= 1 &&
            iz <= sc.nbz - 2) {
            f = 0;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy) {
                    const int row = sc.cbase + (iz + dz) * sc.nbxy + (iy + dy) * sc.nbx;
                    if (wcs[row + ix + 2] > wcs[row + ix - 1]) f = 1;
                }
        }
        near_wall[sc.cbase + b] = f;
    }
}

template <class R, class RN>
__device__ __forceinline__ const SceneDev<R, RN>& scene_ref(const PassArgs<R, RN>& a, int pid) {
    return a.sc[a.nscene > 1 ? scene_of(a.sc, a.nscene, pid) : 0];
}

#define MPS_INF_SKIP(a, v) ((a).skip ? (v) : R(INFINITY))

// a near flag (near_wall, near_m) of the bucket of walk context c; a null table is "near"
template <class R, class RN>
__device__ __forceinline__ bool near_flag(const int8_t* f, const SceneDev<R, RN>& sc,
                                          const RowCtx<R>& c) {
    return !f || __ldg(f + sc.cbase + c.iz * sc.nbxy + c.iy * sc.nbx + c.ix) != 0;
}

// Phase 1 of a neighbour pass: the fluid neighbours j != s with d2 <= thr, in visiting
// order, into the slot's list. Returns the neighbour count (may exceed nbK).
template <class R, class RN, bool COUNT = false>
__device__ __forceinline__ int build_list(const PassArgs<R, RN>& a, const SceneDev<R, RN>& sc,
                                          const RowCtx<R>& c, int s, R x, R y, R z, R thr, R B,
                                          int* ncand = nullptr) {
    int cnt = 0;
    int* __restrict__ nb = a.nb;
    const V4<R>* __restrict__ posf = a.posf;
    const int nF = a.nF, K = a.nbK;
    for_fluid_ranges(sc, a.csr, c, B, [&](int lo, int hi) {
        if (COUNT) *ncand += hi - lo;
        // four independent loads in flight before the first test (latency, not bandwidth,
        // bounds this loop), a short row's included: past the row's end the particle itself
        // pads the batch and visit() rejects it; candidates are tested and appended in
        // visiting order
        auto visit = [&](const V4<R>& q) {
            R dx = q.x - x, dy = q.y - y, dz = q.z - z;
            const int j = w_slot(q.w);
            if (j != s && dot3(dx, dy, dz, dx, dy, dz) <= thr) {
                if (cnt < K) nb[list_at(s, cnt, K)] = j;
                ++cnt;
            }
        };
        const V4<R> self{x, y, z, slot_w(s, R(0))};
        for (int k = lo; k < hi; k += 4) {
            const V4<R> q0 = ldg4(posf + k);
            const V4<R> q1 = k + 1 < hi ? ldg4(posf + k + 1) : self,
                        q2 = k + 2 < hi ? ldg4(posf + k + 2) : self,
                        q3 = k + 3 < hi ? ldg4(posf + k + 3) : self;
            visit(q0);
            visit(q1);
            visit(q2);
            visit(q3);
        }
    });
    return cnt;
}

// ---------------------------------------------------------------------------------------
// shared-memory staging of a block's fluid neighbourhood
// ---------------------------------------------------------------------------------------
// A block's slots are consecutive in bucket-major order, so its particles lie in a few
// x-adjacent buckets, and the candidates all of them visit lie in a small set of fine rows.
// stage_fluid copies those rows' ranges of posf (contiguous per fine row) into shared memory
// with coalesced warp loads, optionally with each candidate's velocity gathered once for the
// whole block, and builds a table of the staged index of every fine cell start. Each
// particle then walks its own rows (for_fluid_rows, the same geometry as the global walk)
// out of shared memory: the same candidates in the same order, so the sums are unchanged.
//
// The staged rows are the union of the particles' fine planes (exact, from their own walk
// bounds) and, per row, the fine x range reached from the box around the particles' float
// coordinates. Every step of the row geometry is monotone in the coordinates, so a box
// corner is never nearer than a particle inside it and the box range covers each
// particle's own range for that row. Blocks whose rows do not fit (particles in two bucket
// rows, more than kStageSpan buckets along x, or more candidates than the staging
// capacity) walk global memory instead, decided uniformly for the block.
constexpr int kStageRows = 81;                     // 9 x 9 fine rows
constexpr int kStageSpan = 8;                      // buckets along x, max - min
constexpr int kStageCols = 3 * kStageSpan + 10;    // fine cells [3 ix_min - 3, 3 ix_max + 5] + end

struct StageHdr {
    int zl, zh, yl, yh;        // union of the particles' fine planes and widest fine rows
    int ixl, ixh;              // bucket x range of the particles
    unsigned box[6];           // x0, x1, y0, y1, z0, z1 as order-preserving integers
    int smin, smax;            // scenes of the particles
    int nrow, ny, fx0, ncol;   // rows staged, rows per plane, first fine x, table columns
    int total;                 // candidates staged
    int xl[kStageRows], xh[kStageRows];  // fine x range staged per row
    int rs[kStageRows];        // posf index of each row's first staged candidate
    int base[kStageRows + 1];  // staged index of each row's first candidate
    int tab[kStageRows * kStageCols];  // staged index of each fine cell start
};

__device__ __forceinline__ unsigned ord_bits(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_float(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}
// distance from [v0, v1] to fine cell f along one axis (fine_gap of the nearer end)
__device__ __forceinline__ float fine_gap_box(float v0, float v1, int f, float hf) {
    const float lo = float(f - 3) * hf;
    return fmaxf(fmaxf(lo - v1, v0 - (lo + hf)), 0.0f);
}

template <class R> __host__ __device__ constexpr size_t stage_smem_bytes(int cap, bool vel) {
    return ((sizeof(StageHdr) + 15) / 16) * 16 + size_t(cap) * sizeof(V4<R>) * (vel ? 2 : 1);
}

// Stage the block's neighbourhood (every thread of the block calls this). `act`: this
// thread holds a particle of scene `scene` whose walk context is `c`; bsel(scene) gives the
// walk bound B (radius plus margin, squared) of the pass. Returns true (uniformly) when the
// stage was built; spos (and svel) then hold the candidates.
template <class R, class RN, bool SVEL, class BSel>
__device__ bool stage_fluid(const PassArgs<R, RN>& a, StageHdr& h, V4<R>* spos, V4<R>* svel,
                            int cap, bool act, int scene, const RowCtx<R>& c, BSel&& bsel) {
    const int tid = threadIdx.x, nth = blockDim.x;
    if (tid == 0) {
        h.zl = h.yl = h.ixl = h.smin = INT_MAX;
        h.zh = h.yh = h.ixh = h.smax = INT_MIN;
        h.box[0] = h.box[2] = h.box[4] = 0xffffffffu;
        h.box[1] = h.box[3] = h.box[5] = 0u;
    }
    __syncthreads();
    if (act) {
        const SceneDev<R, RN>& sc = a.sc[scene];
        const float b = float(bsel(sc)), ih = sc.ihf, s = sqrtf(b);
        atomicMin(&h.zl, fine_at(c.rz - s, ih, 3 * c.iz - 3));
        atomicMax(&h.zh, fine_at(c.rz + s, ih, 3 * c.iz - 3));
        atomicMin(&h.yl, fine_at(c.ry - s, ih, 3 * c.iy - 3));
        atomicMax(&h.yh, fine_at(c.ry + s, ih, 3 * c.iy - 3));
        atomicMin(&h.ixl, c.ix);
        atomicMax(&h.ixh, c.ix);
        atomicMin(&h.box[0], ord_bits(c.rx));
        atomicMax(&h.box[1], ord_bits(c.rx));
        atomicMin(&h.box[2], ord_bits(c.ry));
        atomicMax(&h.box[3], ord_bits(c.ry));
        atomicMin(&h.box[4], ord_bits(c.rz));
        atomicMax(&h.box[5], ord_bits(c.rz));
        atomicMin(&h.smin, scene);
        atomicMax(&h.smax, scene);
    }
    __syncthreads();
    if (h.smax < 0 || h.smin != h.smax) return false;
    const int ny = h.yh - h.yl + 1, nrow = (h.zh - h.zl + 1) * ny;
    if (nrow > kStageRows || h.ixh - h.ixl > kStageSpan) return false;
    const SceneDev<R, RN>& sc = a.sc[h.smin];
    const int fx0 = 3 * h.ixl - 3, ncol = 3 * (h.ixh - h.ixl) + 10;
    const int nfx = 3 * sc.nbx, nfxy = 9 * sc.nbxy;
    // the fine x range of each row reached from the box of the particles
    for (int r = tid; r < nrow; r += nth) {
        const int fz = h.zl + r / ny, fy = h.yl + r % ny;
        const float b = float(bsel(sc)), hf = sc.hf, ih = sc.ihf;
        const float gz = fine_gap_box(ord_float(h.box[4]), ord_float(h.box[5]), fz, hf);
        const float bz = fmaxf(b - gz * gz, 0.0f);
        const float gy = fine_gap_box(ord_float(h.box[2]), ord_float(h.box[3]), fy, hf);
        const float sx = sqrtf(fmaxf(bz - gy * gy, 0.0f));
        const float lo = fmaf(ord_float(h.box[0]) - sx, ih, 3.0f);
        const float hi = fmaf(ord_float(h.box[1]) + sx, ih, 3.0f);
        const int fxh = 3 * h.ixh - 3;
        h.xl[r] = int(fminf(fmaxf(lo, float(fx0)), float(fx0 + 8)));
        h.xh[r] = int(fminf(fmaxf(hi, float(fxh)), float(fxh + 8)));
    }
    __syncthreads();
    // raw posf index of the fine cell starts the rows' ranges need
    for (int e = tid; e < nrow * ncol; e += nth) {
        const int r = e / ncol, k = e - r * ncol;
        if (k >= h.xl[r] - fx0 && k <= h.xh[r] + 1 - fx0) {
            const int fz = h.zl + r / ny, fy = h.yl + r % ny;
            h.tab[r * ncol + k] = __ldg(a.csr + sc.fbase + fz * nfxy + fy * nfx + fx0 + k);
        }
    }
    __syncthreads();
    if (tid < 32) {  // staged bases: exclusive scan of the row counts in row order
        const int lane = tid, per = (nrow + 31) / 32;
        int sum = 0;
        for (int q = 0; q < per; ++q) {
            const int r = lane * per + q;
            if (r < nrow) {
                const int lo = h.tab[r * ncol + h.xl[r] - fx0];
                h.rs[r] = lo;
                sum += h.tab[r * ncol + h.xh[r] + 1 - fx0] - lo;
            }
        }
        int inc = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        int run = inc - sum;
        for (int q = 0; q < per; ++q) {
            const int r = lane * per + q;
            if (r < nrow) {
                h.base[r] = run;
                run += h.tab[r * ncol + h.xh[r] + 1 - fx0] - h.rs[r];
            }
        }
        if (lane == 31) {
            h.base[nrow] = inc;
            h.total = inc;
            h.nrow = nrow;
            h.ny = ny;
            h.fx0 = fx0;
            h.ncol = ncol;
        }
    }
    __syncthreads();
    if (h.total > cap) return false;
    for (int e = tid; e < nrow * ncol; e += nth) {
        const int r = e / ncol, k = e - r * ncol;
        if (k >= h.xl[r] - fx0 && k <= h.xh[r] + 1 - fx0)
            h.tab[r * ncol + k] = h.base[r] + (h.tab[r * ncol + k] - h.rs[r]);
    }
    const int lane = tid & 31;
    for (int r = tid >> 5; r < nrow; r += nth >> 5) {
        const int n = h.base[r + 1] - h.base[r];
        const V4<R>* __restrict__ src = a.posf + h.rs[r];
        V4<R>* dst = spos + h.base[r];
        for (int k = lane; k < n; k += 32) {
            const V4<R> q = ldg4(src + k);
            dst[k] = q;
            if (SVEL) svel[h.base[r] + k] = ldg4(a.vel + w_slot(q.w));
        }
    }
    __syncthreads();
    return true;
}

// the staged range [lo, hi) of fine row (fz, fy), cells [xl, xh]
__device__ __forceinline__ void staged_range(const StageHdr& h, int fz, int fy, int xl, int xh,
                                             int& lo, int& hi) {
    const int* t = h.tab + ((fz - h.zl) * h.ny + (fy - h.yl)) * h.ncol - h.fx0;
    lo = t[xl];
    hi = t[xh + 1];
}

// state of a slot in a recorded step, kept in the w component of the pre-clamp velocity
constexpr int kTapeOk = 0, kTapeClamped = 1, kTapeDeleted = 2, kTapeDead = 3;

// the velocity a kick produced before ChkPcl (kernel.cu:481-513) and what ChkPcl will do
// with it: delete the particle (position outside the box) or clamp |u| to umax
template <class R, class RN>
__device__ __forceinline__ void tape_record(const PassArgs<R, RN>& a, const SceneDev<R, RN>& sc,
                                            int s, R x, R y, R z, R ux, R uy, R uz) {
    int st = kTapeDeleted;
    if (x < sc.hi[0] && x > sc.lo[0] && y < sc.hi[1] && y > sc.lo[1] && z < sc.hi[2] &&
        z > sc.lo[2])
        st = sqrtR(dot3(ux, uy, uz, ux, uy, uz)) > sc.umax ? kTapeClamped : kTapeOk;
    a.tape_pre[s] = V4<R>{ux, uy, uz, R(st)};
}

// Pass A's candidate walk for one particle: each candidate tested, then the velocity term of
// each neighbour in visiting order; NB candidates' positions and the accepted ones'
// velocities in flight at a time (NB = 2, 4 or 8, MPS_OPT_CANDIDATE_BATCH). ranges(f) hands
// the candidate ranges [lo, hi) to f in visiting order; cand(k) is candidate k's position
// (w = slot), velo(k, j) the velocity of candidate k (slot j). TAPE: the neighbours' slots
// also go to the slot's list.
template <class R, class RN, bool TAPE, bool COUNT, int NB = 4, class Ranges, class Cand,
          class Velo>
__device__ __forceinline__ void visc_walk(const PassArgs<R, RN>& a, const SceneDev<R, RN>& sc, int s,
                                          const V4<R>& p, const V4<R>& v, R& sx, R& sy, R& sz,
                                          int& cf, int& ncand, Ranges&& ranges, Cand&& cand,
                                          Velo&& velo) {
    const R two_l0 = sc.two_l0, r_le = sc.r_le;
    int* __restrict__ nb = a.nb;
    const int nF = a.nF, K = a.nbK;
    auto near = [&](const V4<R>& q, int j, R& d2) {
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        d2 = dot3(dx, dy, dz, dx, dy, dz);
        return j != s && d2 <= r_le;  // dist <= r
    };
    auto add = [&](R d2, const V4<R>& u, int j) {
        R d = sqrtR(d2);
        R w = two_l0 / (d2 * d);
        sx = fmaR(u.x - v.x, w, sx);
        sy = fmaR(u.y - v.y, w, sy);
        sz = fmaR(u.z - v.z, w, sz);
        if (TAPE && cf < K) nb[list_at(s, cf, K)] = j;
        ++cf;
    };
    const V4<R> z4{R(0), R(0), R(0), R(0)};
    // a short row's candidates are loaded together too: a batch past the row's end is
    // padded with the particle itself, which near() rejects
    const V4<R> self{p.x, p.y, p.z, slot_w(s, R(0))};
    ranges([&](int lo, int hi) {
        if (COUNT) ncand += hi - lo;
        for (int k = lo; k < hi; k += NB) {
            V4<R> q[NB];
            q[0] = cand(k);
#pragma unroll
            for (int t = 1; t < NB; ++t) q[t] = k + t < hi ? cand(k + t) : self;
            int j[NB];
            R e[NB];
            bool ok[NB];
#pragma unroll
            for (int t = 0; t < NB; ++t) {
                j[t] = w_slot(q[t].w);
                ok[t] = near(q[t], j[t], e[t]);
            }
            V4<R> u[NB];
#pragma unroll
            for (int t = 0; t < NB; ++t) u[t] = ok[t] ? velo(k + t, j[t]) : z4;
#pragma unroll
            for (int t = 0; t < NB; ++t)
                if (ok[t]) add(e[t], u[t], j[t]);
        }
    });
}

// diagnostics: add v of every active lane of the warp to *dst with one atomic
__device__ __forceinline__ void warp_add_u64(unsigned long long* dst, int v) {
    const unsigned m = __activemask();
    const unsigned tot = __reduce_add_sync(m, unsigned(v));
    if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(dst, (unsigned long long)tot);
}

// the rest of pass A for one particle once its fluid sum is known: mirrors (VelM = 0),
// acceleration with gravity, kick/drift (UpPcl1) and ChkPcl, the scratch outputs
template <class R, class RN, bool DIAG, bool TAPE>
__device__ __forceinline__ void pass_a_finish(const PassArgs<R, RN>& a, const SceneDev<R, RN>& sc,
                                              int s, int pid, const V4<R>& p, const V4<R>& v,
                                              const RowCtx<R>& c, R sx, R sy, R sz, int cf) {
    int cm = 0;
    if (TAPE) a.nbcnt[s] = cf;  // the recorded list (complete while cf <= nbK)
    if (near_flag(a.near_m, sc, c))
        visc_sum_mirrors(sc, c, p.x, p.y, p.z, v.x, v.y, v.z, a.m, MPS_INF_SKIP(a, sc.skip_r), sx,
                         sy, sz, cm);
    R ax = fmaR(sc.kn, sx, sc.g[0]), ay = fmaR(sc.kn, sy, sc.g[1]), az = fmaR(sc.kn, sz, sc.g[2]);
    R ux = fmaR(ax, sc.dt, v.x), uy = fmaR(ay, sc.dt, v.y), uz = fmaR(az, sc.dt, v.z);
    R x = fmaR(ux, sc.dt, p.x), y = fmaR(uy, sc.dt, p.y), z = fmaR(uz, sc.dt, p.z);
    if (TAPE) tape_record(a, sc, s, x, y, z, ux, uy, uz);
    bool alive = chkpcl(sc, x, y, z, ux, uy, uz);
    if (!alive) {
        x = y = z = ux = uy = uz = R(0);
        atomicAdd(&a.cnt->deleted, 1);
    }
    a.tpos[s] = V4<R>{x, y, z, R(0)};
    a.tvel[s] = V4<R>{ux, uy, uz, R(0)};
    a.ttyp[s] = alive ? int8_t(kFLD) : int8_t(kGST);
    if (DIAG) {
        int32_t* d = a.diag + size_t(pid) * kDiagCols;
        d[DG_VSC_F] = cf;
        d[DG_VSC_M] = cm;
    }
}

template <class R, class RN>
__device__ __forceinline__ void pass_a_unlisted(const PassArgs<R, RN>& a, int s, bool tape) {
    a.tpos[s] = a.pos[s];
    a.tvel[s] = a.vel[s];
    a.ttyp[s] = a.typ[s];
    if (tape) {
        a.tape_pre[s] = V4<R>{R(0), R(0), R(0), R(kTapeDead)};
        a.nbcnt[s] = 0;
    }
}

// pass A: VscTrm (kernel.cu:1013-1119) + UpPcl1/ChkPcl (kernel.cu:1138-1149, 481-513), each
// particle walking its candidates in global memory (posf through L1).
// TAPE (recorded rollouts): also keeps the list length and the velocity before the clamp.
template <class R, class RN, bool DIAG, bool TAPE = false, int NB = 4, bool ALT = false>
__global__ void __launch_bounds__(128, pass_a_blocks<R>(ALT))
    k_pass_a(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    const int nalive = __ldg(a.cs + a.dead);
    if (s >= nalive) {  // unlisted particles are carried over unchanged
        pass_a_unlisted(a, s, TAPE);
        return;
    }
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    V4<R> p = ldg4(a.pos + s), v = ldg4(a.vel + s);
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    R sx = 0, sy = 0, sz = 0;
    int cf = 0, ncand = 0;
    const V4<R>* __restrict__ posf = a.posf;
    const V4<R>* __restrict__ vel = a.vel;
    visc_walk<R, RN, TAPE, DIAG, NB>(
        a, sc, s, p, v, sx, sy, sz, cf, ncand,
        [&](auto&& f) { for_fluid_ranges(sc, a.csr, c, MPS_INF_SKIP(a, sc.skip_r), f); },
        [&](int k) { return ldg4(posf + k); }, [&](int, int j) { return ldg4(vel + j); });
    if (DIAG) warp_add_u64(&a.cnt->work[0], ncand);
    pass_a_finish<R, RN, DIAG, TAPE>(a, sc, s, pid, p, v, c, sx, sy, sz, cf);
}

// pass A with the block's neighbourhood staged in shared memory (stage_fluid): positions,
// and with SVEL the candidates' velocities too. Same walk order and arithmetic as k_pass_a,
// so the results are identical; blocks whose neighbourhood does not fit walk global memory.
template <class R, class RN, bool DIAG, bool SVEL>
__global__ void __launch_bounds__(128) k_pass_a_st(const __grid_constant__ PassArgs<R, RN> a, int cap) {
    extern __shared__ __align__(16) unsigned char stage_mem[];
    StageHdr& h = *reinterpret_cast<StageHdr*>(stage_mem);
    V4<R>* spos = reinterpret_cast<V4<R>*>(stage_mem + ((sizeof(StageHdr) + 15) / 16) * 16);
    V4<R>* svel = spos + cap;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int nalive = __ldg(a.cs + a.dead);
    const bool act = s < a.nF && s < nalive;
    if (s < a.nF && !act) pass_a_unlisted(a, s, false);
    int pid = 0, scene = 0;
    V4<R> p{R(0), R(0), R(0), R(0)}, v = p;
    RowCtx<R> c{};
    if (act) {
        pid = a.pid[s];
        scene = a.nscene > 1 ? scene_of(a.sc, a.nscene, pid) : 0;
        const SceneDev<R, RN>& sc = a.sc[scene];
        p = ldg4(a.pos + s);
        v = ldg4(a.vel + s);
        int ix, iy, iz;
        cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
        c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    }
    auto bsel = [&](const SceneDev<R, RN>& q) { return MPS_INF_SKIP(a, q.skip_r); };
    const bool staged = stage_fluid<R, RN, SVEL>(a, h, spos, svel, cap, act, scene, c, bsel);
    if (DIAG && threadIdx.x == 0 && h.smax >= 0)
        atomicAdd(staged ? &a.cnt->stage_blocks : &a.cnt->unstaged_blocks, 1);
    if (!act) return;
    const SceneDev<R, RN>& sc = a.sc[scene];
    const R B = bsel(sc);
    R sx = 0, sy = 0, sz = 0;
    int cf = 0, ncand = 0;
    if (staged) {
        const V4<R>* __restrict__ vel = a.vel;
        visc_walk<R, RN, false, DIAG>(
            a, sc, s, p, v, sx, sy, sz, cf, ncand,
            [&](auto&& f) {
                for_fluid_rows(sc, c, B, [&](int fz, int fy, int xl, int xh) {
                    int lo, hi;
                    staged_range(h, fz, fy, xl, xh, lo, hi);
                    f(lo, hi);
                });
            },
            [&](int k) { return spos[k]; },
            [&](int k, int j) { return SVEL ? svel[k] : ldg4(vel + j); });
    } else {
        const V4<R>* __restrict__ posf = a.posf;
        const V4<R>* __restrict__ vel = a.vel;
        visc_walk<R, RN, false, DIAG>(
            a, sc, s, p, v, sx, sy, sz, cf, ncand,
            [&](auto&& f) { for_fluid_ranges(sc, a.csr, c, B, f); },
            [&](int k) { return ldg4(posf + k); }, [&](int, int j) { return ldg4(vel + j); });
    }
    if (DIAG) warp_add_u64(&a.cnt->work[0], ncand);
    pass_a_finish<R, RN, DIAG, false>(a, sc, s, pid, p, v, c, sx, sy, sz, cf);
}

// pass B's stores: velocity after ChkCol, pressure from MkPrs's EOS, diagnostics
template <class R, class RN, bool DIAG>
__device__ __forceinline__ void pass_b_store(const PassArgs<R, RN>& a, const SceneDev<R, RN>& sc,
                                             int s, int pid, R wx, R wy, R wz, RN ni,
                                             const int* cnt5) {
    a.tvel[s] = V4<R>{wx, wy, wz, R(0)};
    a.tprs[s] = eos(sc, ni);
    if (DIAG) {
        int32_t* d = a.diag + size_t(pid) * kDiagCols;
        d[DG_COL_F] = cnt5[0];
        d[DG_COL_W] = cnt5[1];
        d[DG_COL_M] = cnt5[2];
        d[DG_PRS_F] = cnt5[3];
        d[DG_PRS_M] = cnt5[4];
        a.ndens[pid] = ni;
    }
}

// Pass B for the rare slot whose list overflowed its capacity: scans the fine rows again and
// finishes the slot. Out of line, and the last thing its caller does: nothing of the caller's
// stays live across the call, so the list path keeps its values in registers (a call that
// returns sums by reference, or has values live across it, puts them in local memory).
template <class R, class RN, bool DIAG>
__device__ __noinline__ void pass_b_long(const PassArgs<R, RN>& a, int s) {
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    const V4<R> p = ldg4(a.pos + s), v = ldg4(a.vel + s);
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    const RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    R wx = v.x, wy = v.y, wz = v.z;
    RN ni = 0;
    int cnt5[5] = {0, 0, 0, 0, 0};
    col_dens_sum<R, RN, true, true>(sc, c, s, p.x, p.y, p.z, v.x, v.y, v.z, a.csr, a.posf, a.vel,
                                    a.wl, a.m, a.skip != 0, wx, wy, wz, ni, cnt5);
    pass_b_store<R, RN, DIAG>(a, sc, s, pid, wx, wy, wz, ni, cnt5);
}

// pass B: ChkCol (kernel.cu:1168-1287) + MkPrs (kernel.cu:1306-1411) at x*; leaves the
// list of fluid neighbours inside max(rp, rlim) for pass C (same positions, same slots)
template <class R, class RN, bool DIAG, bool ALT = false>
__global__ void __launch_bounds__(128, pass_b_blocks<R>(ALT))
    k_pass_b(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    const int nalive = __ldg(a.cs + a.dead);
    if (s >= nalive) {
        a.tvel[s] = a.vel[s];
        a.tprs[s] = R(0);
        return;
    }
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    V4<R> p = ldg4(a.pos + s), v = ldg4(a.vel + s);
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    int ncand = 0;
    const int n = build_list<R, RN, DIAG>(a, sc, c, s, p.x, p.y, p.z, sc.list_thr,
                                          MPS_INF_SKIP(a, sc.skip_rc), &ncand);
    a.nbcnt[s] = n;
    if (DIAG) {
        warp_add_u64(&a.cnt->work[1], ncand);
        warp_add_u64(&a.cnt->work[2], n);
    }
    if (n > a.nbK) {
        pass_b_long<R, RN, DIAG>(a, s);
        return;
    }
    R wx = v.x, wy = v.y, wz = v.z;
    RN ni = 0;
    int cnt5[5] = {0, 0, 0, 0, 0};
    const int* __restrict__ nb = a.nb + list_at(s, 0, a.nbK);
    const V4<R>* __restrict__ pos = a.pos;
    const V4<R>* __restrict__ vel = a.vel;
    const int st = 32;
    const R rlim2 = sc.rlim2, rp_lt = sc.rp_lt, colfac = sc.colfac, rp = sc.rp;
    const RN rp_n = sc.rp_n;
    auto add = [&](int j, const V4<R>& q) {
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 < rlim2) {
            V4<R> u = ldg4(vel + j);
            col_hit(colfac, v.x, v.y, v.z, u.x, u.y, u.z, dx, dy, dz, d2, wx, wy, wz);
            ++cnt5[0];
        }
        if (d2 <= rp_lt) {
            dens_add_v(rp, rp_n, d2, ni);
            ++cnt5[3];
        }
    };
    int k = 0;
    for (; k + 4 <= n; k += 4) {
        const int j0 = nb[k * st], j1 = nb[(k + 1) * st], j2 = nb[(k + 2) * st],
                  j3 = nb[(k + 3) * st];
        V4<R> q0 = ldg4(pos + j0), q1 = ldg4(pos + j1), q2 = ldg4(pos + j2), q3 = ldg4(pos + j3);
        add(j0, q0);
        add(j1, q1);
        add(j2, q2);
        add(j3, q3);
    }
    for (; k < n; ++k) {
        const int j = nb[k * st];
        add(j, ldg4(pos + j));
    }
    col_dens_walls_mirrors<R, RN, true, true>(sc, c, p.x, p.y, p.z, v.x, v.y, v.z, a.wl, a.m,
                                              a.skip != 0, wx, wy, wz, ni, cnt5,
                                              near_flag(a.near_wall, sc, c),
                                              near_flag(a.near_m, sc, c));
    pass_b_store<R, RN, DIAG>(a, sc, s, pid, wx, wy, wz, ni, cnt5);
}

// pass C's end for one slot: acceleration from the gradient sums, UpPcl2 (kick and drift),
// ChkPcl, stores and diagnostics
template <class R, class RN, bool DIAG, bool TAPE, class G>
__device__ __forceinline__ void pass_c_finish(const PassArgs<R, RN>& a, const SceneDev<R, RN>& sc,
                                              int s, int pid, const V4<R>& p, R pi, const G& g,
                                              int cf, int cm) {
    V4<R> v = a.tvel[s];
    R ax, ay, az;
    if (!grad_acc(sc, g, ax, ay, az)) {
        ax = v.x;
        ay = v.y;
        az = v.z;
    }
    R ux = fmaR(ax, sc.dt, v.x), uy = fmaR(ay, sc.dt, v.y), uz = fmaR(az, sc.dt, v.z);
    R x = fmaR(ax * sc.dt, sc.dt, p.x), y = fmaR(ay * sc.dt, sc.dt, p.y),
      z = fmaR(az * sc.dt, sc.dt, p.z);
    a.pav[s] = a.pav[s] + pi;
    if (TAPE) tape_record(a, sc, s, x, y, z, ux, uy, uz);
    bool alive = chkpcl(sc, x, y, z, ux, uy, uz);
    if (!alive) {
        x = y = z = ux = uy = uz = R(0);
        atomicAdd(&a.cnt->deleted, 1);
    }
    a.tpos[s] = V4<R>{x, y, z, R(0)};
    a.tvel[s] = V4<R>{ux, uy, uz, R(0)};
    a.ttyp[s] = alive ? int8_t(kFLD) : int8_t(kGST);
    if (DIAG) {
        int32_t* d = a.diag + size_t(pid) * kDiagCols;
        d[DG_GRD_F] = cf;
        d[DG_GRD_M] = cm;
    }
}

// Pass C for a slot whose list overflowed its capacity: the fine-row scan, then the slot's
// end; out of line and a tail call, like pass_b_long
template <class R, class RN, bool DIAG, bool TAPE, class G>
__device__ __noinline__ void pass_c_long(const PassArgs<R, RN>& a, int s) {
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    const V4<R> p = ldg4(a.pos + s);
    const R pi = a.tprs[s];
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    const RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    G g;
    int cf = 0, cm = 0;
    grad_sum(sc, c, s, pid - sc.pbase, p.x, p.y, p.z, pi, a.csr, a.posf, a.tprs, a.m,
             a.skip != 0, g, cf, cm);
    pass_c_finish<R, RN, DIAG, TAPE>(a, sc, s, pid, p, pi, g, cf, cm);
}

// pass C: PrsGrdTrm (kernel.cu:1651-1794) + UpPcl2/ChkPcl (kernel.cu:1815-1829), walking
// the neighbour lists pass B left. TAPE: also keeps the velocity before the clamp. CORR: the
// corrected-matrix PrsGrdTrm (kernel.cu:1435-1648); where its moment matrix is all zero the
// reference leaves in d_Acc the velocity ChkCol stored there (kernel.cu:1275, 1620), which
// UpPcl2 then applies as the acceleration: the velocity after pass B, as here.
template <class R, class RN, bool DIAG, bool TAPE = false, bool CORR = false, bool ALT = false>
__global__ void __launch_bounds__(128, pass_c_blocks<R>(ALT, CORR))
    k_pass_c(const __grid_constant__ PassArgs<R, RN> a) {
    using G = typename std::conditional<CORR, GradCorr<R>, GradPlain<R>>::type;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    const int nalive = __ldg(a.cs + a.dead);
    if (s >= nalive) {
        a.tpos[s] = a.pos[s];
        a.ttyp[s] = a.typ[s];
        if (TAPE) a.tape_pre[s] = V4<R>{R(0), R(0), R(0), R(kTapeDead)};
        return;
    }
    const int n = a.nbcnt[s];
    if (n > a.nbK) {
        pass_c_long<R, RN, DIAG, TAPE, G>(a, s);
        return;
    }
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    V4<R> p = ldg4(a.pos + s);
    const R pi = a.tprs[s];
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    G g;
    int cf = 0, cm = 0;
    const int* __restrict__ nb = a.nb + list_at(s, 0, a.nbK);
    const V4<R>* __restrict__ pos = a.pos;
    const R* __restrict__ prs = a.tprs;
    const int st = 32;
    const R rp2 = sc.rp2, rp = sc.rp;
    // P_min over the fluid neighbours inside rp (order-free), then the gradient in order
    R pmin = pi;
    // each list entry's position and pressure are loaded together (both depend only on
    // the index), four entries in flight, before the tests that use them
    auto mn = [&](const V4<R>& q, R pj) {
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        if (dot3(dx, dy, dz, dx, dy, dz) < rp2 && pj < pmin) pmin = pj;
    };
    int k = 0;
    for (; k + 4 <= n; k += 4) {
        const int j0 = nb[k * st], j1 = nb[(k + 1) * st], j2 = nb[(k + 2) * st],
                  j3 = nb[(k + 3) * st];
        V4<R> q0 = ldg4(pos + j0), q1 = ldg4(pos + j1), q2 = ldg4(pos + j2), q3 = ldg4(pos + j3);
        const R r0 = __ldg(prs + j0), r1 = __ldg(prs + j1), r2 = __ldg(prs + j2),
                r3 = __ldg(prs + j3);
        mn(q0, r0);
        mn(q1, r1);
        mn(q2, r2);
        mn(q3, r3);
    }
    for (; k < n; ++k) {
        const int j = nb[k * st];
        mn(ldg4(pos + j), __ldg(prs + j));
    }
    auto gr = [&](const V4<R>& q, R pj) {
        R dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 < rp2) {
            R d = sqrtR(d2);
            g.add(wei_grad(d, rp) / d2, pj - pmin, dx, dy, dz);
            ++cf;
        }
    };
    for (k = 0; k + 4 <= n; k += 4) {
        const int j0 = nb[k * st], j1 = nb[(k + 1) * st], j2 = nb[(k + 2) * st],
                  j3 = nb[(k + 3) * st];
        V4<R> q0 = ldg4(pos + j0), q1 = ldg4(pos + j1), q2 = ldg4(pos + j2), q3 = ldg4(pos + j3);
        const R r0 = __ldg(prs + j0), r1 = __ldg(prs + j1), r2 = __ldg(prs + j2),
                r3 = __ldg(prs + j3);
        gr(q0, r0);
        gr(q1, r1);
        gr(q2, r2);
        gr(q3, r3);
    }
    for (; k < n; ++k) {
        const int j = nb[k * st];
        gr(ldg4(pos + j), __ldg(prs + j));
    }
    if (near_flag(a.near_m, sc, c))
        grad_sum_mirrors(sc, c, pid - sc.pbase, p.x, p.y, p.z, pmin, a.m, a.skip != 0, g, cm);
    pass_c_finish<R, RN, DIAG, TAPE>(a, sc, s, pid, p, pi, g, cf, cm);
}

// The warp's mirrors take consecutive places in the raw list, reserved with one atomic per
// warp (the list's order does not matter: the mirror bucket build sorts by bucket and slot).
// Every lane of the warp calls this.
template <class R, class RN, bool TAPE>
__device__ __forceinline__ void gen_reserve_emit(const PassArgs<R, RN>& a, const MirrorPlan<R>& pl,
                                                 int m, R x, R y, R z, R P, int slot_base) {
    const int lane = threadIdx.x & 31;
    int incl = m;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int tot = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 31 && tot > 0) base = atomicAdd(&a.cnt->mirror_raw, tot);
    base = __shfl_sync(0xffffffffu, base, 31) + incl - m;
    if (m > 0) emit_mirrors<R, RN, TAPE>(pl, x, y, z, P, slot_base, a.wl, a.out, a.cnt, base);
}

// GenMRR_nonslip + MRRinout for every FLD slot of (gpos, gprs, gtyp): the second generation
// of a step (x*, P after pass B) and the first generation of the next one (x^{n+1}, P after
// pass C). Near-wall particles are a thin layer, so this runs as a light kernel of its own
// instead of stretching the neighbour passes. With gprs null a mirror's pressure field holds
// its owner's slot instead, for k_mirror_prs to replace once the pressures exist: the
// positions of the second generation need only x*, so they are made beside pass B.
template <class R, class RN, bool DIAG, bool TAPE = false>
__global__ void __launch_bounds__(128, min_blocks<R>(10)) k_gen_cull(const __grid_constant__ PassArgs<R, RN> a, const V4<R>* gpos,
                                                  const R* gprs, const int8_t* gtyp) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    MirrorPlan<R> pl;
    pl.nreg = 0;
    pl.corner = -1;
    int m = 0, pid = 0;
    V4<R> p{R(0), R(0), R(0), R(0)};
    R P = R(0);
    if (s < a.nF && gtyp[s] == kFLD) {  // every lane stays for the warp's reservation
        pid = a.pid[s];
        const SceneDev<R, RN>& sc = scene_ref(a, pid);
        p = gpos[s];
        int ix, iy, iz;
        cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
        int nw = 0;
        // no wall in the 27 buckets around: no wall within r, no mirror (the common case)
        if (__ldg(a.near_wall + sc.cbase + iz * sc.nbxy + iy * sc.nbx + ix)) {
            RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
            nw = plan_mirrors(sc, c, p.x, p.y, p.z, a.wl, a.skip != 0, pl);
            m = count_mirrors<R, RN>(pl, p.x, p.y, p.z, a.wl, a.cnt);
            P = gprs ? gprs[s] : slot_w(s, R(0));
        }
        if (DIAG) a.diag[size_t(pid) * kDiagCols + DG_GEN_W] = nw;
    }
    gen_reserve_emit<R, RN, TAPE>(a, pl, m, p.x, p.y, p.z, P, pid * kNumMRR);
}

// The pressures of a mirror generation made without them (k_gen_cull with gprs null), once
// they exist: each bucketed mirror's owner slot, kept in its pressure field, becomes that
// slot's pressure (PrsM = Prs of the owner, as the generation writes it directly). Only the
// mirrors of the table's live buckets are read; a slot outside [0, nF) is left alone.
template <class R>
__global__ void k_mirror_prs(const int* __restrict__ mcs, int dead, V4<R>* __restrict__ mpos,
                             const R* __restrict__ prs, int nF) {
    const int n = __ldg(mcs + dead);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int s = w_slot(mpos[k].w);
        if (s >= 0 && s < nF) mpos[k].w = prs[s];
    }
}

// ---------------------------------------------------------------------------------------
// one reference method per launch (mps_phase); state is updated in place like the
// reference's device arrays
// ---------------------------------------------------------------------------------------
template <class R, class RN, bool DIAG>
__global__ void __launch_bounds__(128) k_ph_vsc(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF || a.typ[s] != kFLD) return;
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    V4<R> p = ldg4(a.pos + s), v = ldg4(a.vel + s);
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    R sx = 0, sy = 0, sz = 0;
    int cf = 0, cm = 0;
    visc_sum(sc, c, s, p.x, p.y, p.z, v.x, v.y, v.z, a.csr, a.posf, a.vel, a.m,
             MPS_INF_SKIP(a, sc.skip_r), sx, sy, sz, cf, cm);
    a.acc[s] = V4<R>{fmaR(sc.kn, sx, sc.g[0]), fmaR(sc.kn, sy, sc.g[1]), fmaR(sc.kn, sz, sc.g[2]),
                     R(0)};
    if (DIAG) {
        int32_t* d = a.diag + size_t(pid) * kDiagCols;
        d[DG_VSC_F] = cf;
        d[DG_VSC_M] = cm;
    }
}

template <class R, class RN>
__global__ void k_ph_uppcl1(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF || a.typ[s] != kFLD) return;
    const SceneDev<R, RN>& sc = scene_ref(a, a.pid[s]);
    V4<R> p = a.pos[s], v = a.vel[s], ac = a.acc[s];
    R ux = fmaR(ac.x, sc.dt, v.x), uy = fmaR(ac.y, sc.dt, v.y), uz = fmaR(ac.z, sc.dt, v.z);
    R x = fmaR(ux, sc.dt, p.x), y = fmaR(uy, sc.dt, p.y), z = fmaR(uz, sc.dt, p.z);
    if (chkpcl(sc, x, y, z, ux, uy, uz)) {
        a.pos[s] = V4<R>{x, y, z, R(0)};
        a.vel[s] = V4<R>{ux, uy, uz, R(0)};
    } else {
        a.typ[s] = kGST;
        a.pos[s] = V4<R>{0, 0, 0, 0};
        a.vel[s] = V4<R>{0, 0, 0, 0};
        a.prs[s] = R(0);
        atomicAdd(&a.cnt->deleted, 1);
    }
    a.acc[s] = V4<R>{0, 0, 0, 0};
}

template <class R, class RN, bool DIAG>
__global__ void __launch_bounds__(128) k_ph_col(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF || a.typ[s] != kFLD) return;
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    V4<R> p = ldg4(a.pos + s), v = ldg4(a.vel + s);
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    R wx = v.x, wy = v.y, wz = v.z;
    RN ni = 0;
    int cnt5[5] = {0, 0, 0, 0, 0};
    col_dens_sum<R, RN, true, false>(sc, c, s, p.x, p.y, p.z, v.x, v.y, v.z, a.csr, a.posf, a.vel,
                                     a.wl, a.m, a.skip != 0, wx, wy, wz, ni, cnt5);
    a.tvel[s] = V4<R>{wx, wy, wz, R(0)};
    if (DIAG) {
        int32_t* d = a.diag + size_t(pid) * kDiagCols;
        d[DG_COL_F] = cnt5[0];
        d[DG_COL_W] = cnt5[1];
        d[DG_COL_M] = cnt5[2];
    }
}

// d_UpChkCol (kernel.cu:1281-1287): Acc holds the corrected velocity, Vel = Acc
template <class R, class RN>
__global__ void k_ph_upchkcol(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF || a.typ[s] != kFLD) return;
    V4<R> w = a.tvel[s];
    a.acc[s] = w;
    a.vel[s] = w;
}

template <class R, class RN, bool DIAG>
__global__ void __launch_bounds__(128) k_ph_prs(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF || a.typ[s] != kFLD) return;
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    V4<R> p = ldg4(a.pos + s);
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    R wx = 0, wy = 0, wz = 0;
    RN ni = 0;
    int cnt5[5] = {0, 0, 0, 0, 0};
    col_dens_sum<R, RN, false, true>(sc, c, s, p.x, p.y, p.z, R(0), R(0), R(0), a.csr, a.posf,
                                     a.vel, a.wl, a.m, a.skip != 0, wx, wy, wz, ni, cnt5);
    a.prs[s] = eos(sc, ni);
    if (DIAG) {
        int32_t* d = a.diag + size_t(pid) * kDiagCols;
        d[DG_PRS_F] = cnt5[3];
        d[DG_PRS_M] = cnt5[4];
        a.ndens[pid] = ni;
    }
}

template <class R, class RN, bool DIAG, bool CORR = false>
__global__ void __launch_bounds__(128) k_ph_grd(const __grid_constant__ PassArgs<R, RN> a) {
    using G = typename std::conditional<CORR, GradCorr<R>, GradPlain<R>>::type;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF || a.typ[s] != kFLD) return;
    const int pid = a.pid[s];
    const SceneDev<R, RN>& sc = scene_ref(a, pid);
    V4<R> p = ldg4(a.pos + s);
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    G g;
    int cf = 0, cm = 0;
    grad_sum(sc, c, s, pid - sc.pbase, p.x, p.y, p.z, a.prs[s], a.csr, a.posf, a.prs, a.m,
             a.skip != 0, g, cf, cm);
    R ax, ay, az;
    if (grad_acc(sc, g, ax, ay, az)) a.acc[s] = V4<R>{ax, ay, az, R(0)};  // else d_Acc stays
    if (DIAG) {
        int32_t* d = a.diag + size_t(pid) * kDiagCols;
        d[DG_GRD_F] = cf;
        d[DG_GRD_M] = cm;
    }
}

template <class R, class RN>
__global__ void k_ph_uppcl2(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nF) return;
    if (a.typ[s] == kFLD) {
        const SceneDev<R, RN>& sc = scene_ref(a, a.pid[s]);
        V4<R> p = a.pos[s], v = a.vel[s], ac = a.acc[s];
        R ux = fmaR(ac.x, sc.dt, v.x), uy = fmaR(ac.y, sc.dt, v.y), uz = fmaR(ac.z, sc.dt, v.z);
        R x = fmaR(ac.x * sc.dt, sc.dt, p.x), y = fmaR(ac.y * sc.dt, sc.dt, p.y),
          z = fmaR(ac.z * sc.dt, sc.dt, p.z);
        a.acc[s] = V4<R>{0, 0, 0, 0};
        a.pav[s] = a.pav[s] + a.prs[s];
        if (chkpcl(sc, x, y, z, ux, uy, uz)) {
            a.pos[s] = V4<R>{x, y, z, R(0)};
            a.vel[s] = V4<R>{ux, uy, uz, R(0)};
        } else {
            a.typ[s] = kGST;
            a.pos[s] = V4<R>{0, 0, 0, 0};
            a.vel[s] = V4<R>{0, 0, 0, 0};
            a.prs[s] = R(0);
            atomicAdd(&a.cnt->deleted, 1);
        }
    } else {
        a.pav[s] = a.pav[s] + a.prs[s];
    }
}

// GenMRR_nonslip without the cull (the cull is MkBkt_MRR's d_MRRinout)
template <class R, class RN, bool DIAG>
__global__ void __launch_bounds__(128) k_ph_gen(const __grid_constant__ PassArgs<R, RN> a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    MirrorPlan<R> pl;
    pl.nreg = 0;
    pl.corner = -1;
    int m = 0, pid = 0;
    V4<R> p{R(0), R(0), R(0), R(0)};
    R P = R(0);
    if (s < a.nF && a.typ[s] == kFLD) {  // every lane stays for the warp's reservation
        pid = a.pid[s];
        const SceneDev<R, RN>& sc = scene_ref(a, pid);
        p = ldg4(a.pos + s);
        int ix, iy, iz;
        cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
        RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
        const int nw = plan_mirrors(sc, c, p.x, p.y, p.z, a.wl, a.skip != 0, pl);
        m = count_mirrors<R, RN>(pl, p.x, p.y, p.z, a.wl, a.cnt);
        P = a.prs[s];
        if (DIAG) a.diag[size_t(pid) * kDiagCols + DG_GEN_W] = nw;
    }
    gen_reserve_emit<R, RN, false>(a, pl, m, p.x, p.y, p.z, P, pid * kNumMRR);
}

// Nearest wall inside r of a mirror over part of its 27 buckets' rows: row ri = 3 (dz + 1)
// + (dy + 1) when ri % 4 == part (for_rows's rows and skipping). Keeps the first nearest
// wall in visiting order: distance, row and wall slot (-1: none).
template <class R, class RN>
__device__ __forceinline__ void nearest_wall_part(const SceneDev<R, RN>& sc, const RowCtx<R>& c,
                                                  R mx, R my, R mz, const WallView<R>& wl, R B,
                                                  int part, R& wd, int& wrow, int& wj) {
#pragma unroll 1
    for (int ri = part; ri < 9; ri += 4) {
        const int dz = ri / 3 - 1, dy = ri % 3 - 1;
        const R ddz = dz < 0 ? c.dzl : (dz > 0 ? c.dzh : R(0));
        const R ddy = dy < 0 ? c.dyl : (dy > 0 ? c.dyh : R(0));
        const R dyz2 = ddy * ddy + ddz * ddz;
        if (dyz2 > B) continue;
        const int jl = (dyz2 + c.dxl * c.dxl <= B) ? c.ix - 1 : c.ix;
        const int jh = (dyz2 + c.dxh * c.dxh <= B) ? c.ix + 1 : c.ix;
        const int row = sc.cbase + (c.iz + dz) * sc.nbxy + (c.iy + dy) * sc.nbx;
        const int lo = __ldg(wl.cs + row + jl), hi = __ldg(wl.cs + row + jh + 1);
        for (int j = lo; j < hi; ++j) {
            V4<R> q = ldg4(wl.pos + j);
            R dx = mx - q.x, dy2 = my - q.y, dz2 = mz - q.z;
            R d2 = dot3(dx, dy2, dz2, dx, dy2, dz2);
            if (d2 <= sc.r_le) {  // dist <= r
                R d = sqrtR(d2);
                if (d < wd) {
                    wd = d;
                    wrow = ri;
                    wj = j;
                }
            }
        }
    }
}

// d_MRRinout (kernel.cu:932-985) over the raw mirrors; a culled mirror's slot becomes
// negative. Four lanes share a mirror, each walking a quarter of its rows; the group then
// keeps the smallest distance, on ties the earlier row, which is the wall the sequential
// walk keeps (the first nearest one found).
template <class R, class RN>
__global__ void k_ph_cull(const __grid_constant__ PassArgs<R, RN> a) {
    const int n = min(a.cnt->mirror_raw, a.out.cap);
    const int part = threadIdx.x & 3;
    const int groups = (gridDim.x * blockDim.x) >> 2;
    const int nround = (n + groups - 1) / groups * groups;  // every lane loops alike
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 2; t < nround; t += groups) {
        const int sl = t < n ? a.out.slot[t] : -1;
        R wd = R(0);
        int wrow = 9, wj = -1;
        V4<R> q{R(0), R(0), R(0), R(0)};
        const SceneDev<R, RN>* scp = a.sc;
        if (sl >= 0) {
            scp = &a.sc[a.nscene > 1 ? scene_of(a.sc, a.nscene, sl / kNumMRR) : 0];
            q = a.out.pos[t];
            int ix, iy, iz;
            if (!cell_of(*scp, q.x, q.y, q.z, ix, iy, iz) && part == 0) atomicAdd(&a.cnt->err_cell, 1);
            const RowCtx<R> c = row_ctx(*scp, q.x, q.y, q.z, ix, iy, iz);
            wd = scp->wall_dist0;
            nearest_wall_part(*scp, c, q.x, q.y, q.z, a.wl, a.skip != 0 ? scp->skip_r : R(INFINITY),
                              part, wd, wrow, wj);
        }
        for (int o = 1; o <= 2; o <<= 1) {
            const R od = __shfl_xor_sync(0xffffffffu, wd, o);
            const int orow = __shfl_xor_sync(0xffffffffu, wrow, o);
            const int oj = __shfl_xor_sync(0xffffffffu, wj, o);
            if (oj >= 0 && (wj < 0 || od < wd || (od == wd && orow < wrow))) {
                wd = od;
                wrow = orow;
                wj = oj;
            }
        }
        if (part == 0 && sl >= 0 && wj >= 0) {
            const V4<R> w = ldg4(a.wl.pos + wj), nv = ldg4(a.wl.nrm + wj);
            if (dot3(q.x - w.x, q.y - w.y, q.z - w.z, nv.x, nv.y, nv.z) >= R(0))
                a.out.slot[t] = -1 - sl;
        }
    }
}

// ---------------------------------------------------------------------------------------
// moving walls: the reference declares a rotating wall (w, wallangle, rot_rad,
// class.cuh:117-121) and asks for Surface_Edge every step once walls move (kernel.cu:1879),
// but never moves one. Here OBJ and OBJ2 can follow a prescribed rigid motion.
// ---------------------------------------------------------------------------------------
// q <- qs q and t <- t + vdt for every moving type (one thread, fixed operation order)
static __global__ void k_motion_advance(WallMotion* m) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int k = 0; k < 2; ++k) {
        WallMotion& w = m[k];
        if (w.type == 0) continue;
        double r[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                r[3 * i + j] = (w.qs[3 * i] * w.q[j] + w.qs[3 * i + 1] * w.q[3 + j]) +
                               w.qs[3 * i + 2] * w.q[6 + j];
        for (int i = 0; i < 9; ++i) w.q[i] = r[i];
        for (int d = 0; d < 3; ++d) w.t[d] = w.t[d] + w.vdt[d];
    }
}

// the moving walls' place, normal and velocity from their reference state (x0, n0: double
// SoA of the nW walls in load order)
template <class R>
__global__ void k_move_walls(const WallMotion* __restrict__ m, int nW,
                             const int8_t* __restrict__ typ, const double* __restrict__ x0,
                             const double* __restrict__ n0, V4<R>* pos, V4<R>* nrm, V4<R>* vel) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nW) return;
    const int ty = typ[t];
    const int k = (m[0].type != 0 && ty == m[0].type) ? 0 : ((m[1].type != 0 && ty == m[1].type) ? 1 : -1);
    if (k < 0) return;
    const WallMotion& w = m[k];
    const double dx = x0[t] - w.c[0], dy = x0[nW + t] - w.c[1], dz = x0[2 * size_t(nW) + t] - w.c[2];
    const double rx = (w.q[0] * dx + w.q[1] * dy) + w.q[2] * dz;
    const double ry = (w.q[3] * dx + w.q[4] * dy) + w.q[5] * dz;
    const double rz = (w.q[6] * dx + w.q[7] * dy) + w.q[8] * dz;
    const double ax = n0[t], ay = n0[nW + t], az = n0[2 * size_t(nW) + t];
    pos[t] = V4<R>{R((w.c[0] + w.t[0]) + rx), R((w.c[1] + w.t[1]) + ry), R((w.c[2] + w.t[2]) + rz),
                   R(0)};
    nrm[t] = V4<R>{R((w.q[0] * ax + w.q[1] * ay) + w.q[2] * az),
                   R((w.q[3] * ax + w.q[4] * ay) + w.q[5] * az),
                   R((w.q[6] * ax + w.q[7] * ay) + w.q[8] * az), R(0)};
    vel[t] = V4<R>{R(w.v[0] + (w.w[1] * rz - w.w[2] * ry)), R(w.v[1] + (w.w[2] * rx - w.w[0] * rz)),
                   R(w.v[2] + (w.w[0] * ry - w.w[1] * rx)), R(0)};
}

// reference state of the walls of one type, taken when its motion is set
template <class R>
__global__ void k_motion_snapshot(int nW, const int8_t* __restrict__ typ, int type,
                                  const V4<R>* __restrict__ pos, const V4<R>* __restrict__ nrm,
                                  double* x0, double* n0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nW || typ[t] != type) return;
    const V4<R> p = pos[t], n = nrm[t];
    x0[t] = double(p.x); x0[nW + t] = double(p.y); x0[2 * size_t(nW) + t] = double(p.z);
    n0[t] = double(n.x); n0[nW + t] = double(n.y); n0[2 * size_t(nW) + t] = double(n.z);
}

// d_Surface_Edge (kernel.cu:553-668) over the sorted walls
template <class R, class RN>
__global__ void k_surface_edge(const SceneDev<R, RN>* scs, int nscene, int nW, WallView<R> wl,
                               const int* wid, int8_t* wse) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nW) return;
    const SceneDev<R, RN>& sc = scs[nscene > 1 ? scene_of(scs, nscene, wid[t]) : 0];
    V4<R> p = wl.pos[t], n = wl.nrm[t];
    int8_t ty = wl.typ[t];
    int ix, iy, iz;
    cell_of(sc, p.x, p.y, p.z, ix, iy, iz);
    RowCtx<R> c = row_ctx(sc, p.x, p.y, p.z, ix, iy, iz);
    bool edge = false;
    for_rows(sc, wl.cs, c, R(INFINITY), [&](int j) {
        if (j == t || wl.typ[j] != ty) return;
        V4<R> q = wl.pos[j];
        R dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
        R d2 = dot3(dx, dy, dz, dx, dy, dz);
        if (d2 < sc.edge_r2) {
            V4<R> m = wl.nrm[j];
            if (m.x != n.x || m.y != n.y || m.z != n.z) edge = true;
        }
    });
    wse[t] = edge ? int8_t(kEDGE) : int8_t(0);
}

// ---------------------------------------------------------------------------------------
// state transfer between id order (host layout) and slot order
// ---------------------------------------------------------------------------------------
template <class R> struct IdState {  // SoA, id order, n = all particles; a null array is skipped
    int n;
    R* pos; R* vel; R* acc; R* prs; R* pav; int8_t* typ;
    int* cell;  // bucket index ib of the current position, -1 for GST
};

template <class R, class RN>
__device__ __forceinline__ int local_cell(const SceneDev<R, RN>& sc, R x, R y, R z) {
    int ix = int((x - sc.minc[0]) * sc.dbinv) + 1;
    int iy = int((y - sc.minc[1]) * sc.dbinv) + 1;
    int iz = int((z - sc.minc[2]) * sc.dbinv) + 1;
    return iz * sc.nbxy + iy * sc.nbx + ix;
}

template <class R>
__global__ void k_load_fluid(IdState<R> st, const int* fluid_ids, int nF, V4<R>* pos, V4<R>* vel,
                             V4<R>* acc, R* prs, R* pav, int* pid, int8_t* typ, int use_acc) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const int id = fluid_ids[f];
    const size_t n = st.n;
    pos[f] = V4<R>{st.pos[id], st.pos[n + id], st.pos[2 * n + id], R(0)};
    vel[f] = V4<R>{st.vel[id], st.vel[n + id], st.vel[2 * n + id], R(0)};
    acc[f] = use_acc ? V4<R>{st.acc[id], st.acc[n + id], st.acc[2 * n + id], R(0)}
                     : V4<R>{0, 0, 0, 0};
    prs[f] = st.prs[id];
    pav[f] = st.pav[id];
    pid[f] = id;
    typ[f] = st.typ[id] == kFLD ? int8_t(kFLD) : int8_t(kGST);
}

template <class R>
__global__ void k_load_walls(int n, const R* pos, const R* vel, const R* nrm, const int8_t* ty,
                             const int* wall_ids, int nW, V4<R>* wpos, V4<R>* wvel, V4<R>* wnrm,
                             int* wid, int8_t* wtyp) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nW) return;
    const int id = wall_ids[w];
    const size_t N = n;
    wpos[w] = V4<R>{pos[id], pos[N + id], pos[2 * N + id], R(0)};
    wvel[w] = V4<R>{vel[id], vel[N + id], vel[2 * N + id], R(0)};
    wnrm[w] = V4<R>{nrm[id], nrm[N + id], nrm[2 * N + id], R(0)};
    wid[w] = id;
    wtyp[w] = ty[id];
}

template <class R, class RN>
__global__ void k_store_fluid(IdState<R> st, const SceneDev<R, RN>* scs, int nscene, int nF,
                              const V4<R>* pos, const V4<R>* vel, const V4<R>* acc, const R* prs,
                              const R* pav, const int* pid, const int8_t* typ) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nF) return;
    const int id = pid[s];
    if (st.cell) {
        const SceneDev<R, RN>& sc = scs[nscene > 1 ? scene_of(scs, nscene, id) : 0];
        st.cell[id] = typ[s] == kFLD ? local_cell(sc, pos[s].x, pos[s].y, pos[s].z) : -1;
    }
    const size_t n = st.n;
    if (st.pos) {
        const V4<R> p = pos[s];
        st.pos[id] = p.x; st.pos[n + id] = p.y; st.pos[2 * n + id] = p.z;
    }
    if (st.vel) {
        const V4<R> v = vel[s];
        st.vel[id] = v.x; st.vel[n + id] = v.y; st.vel[2 * n + id] = v.z;
    }
    if (st.acc) {
        const V4<R> a = acc[s];
        st.acc[id] = a.x; st.acc[n + id] = a.y; st.acc[2 * n + id] = a.z;
    }
    if (st.prs) st.prs[id] = prs[s];
    if (st.pav) st.pav[id] = pav[s];
    if (st.typ) st.typ[id] = typ[s];
}

template <class R, class RN>
__global__ void k_store_walls(IdState<R> st, const SceneDev<R, RN>* scs, int nscene, int nW,
                              const V4<R>* pos, const V4<R>* vel, const int* wid,
                              const int8_t* wtyp) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nW) return;
    const int id = wid[w];
    if (st.cell) {
        const SceneDev<R, RN>& sc = scs[nscene > 1 ? scene_of(scs, nscene, id) : 0];
        st.cell[id] = local_cell(sc, pos[w].x, pos[w].y, pos[w].z);
    }
    const size_t n = st.n;
    if (st.pos) {
        const V4<R> p = pos[w];
        st.pos[id] = p.x; st.pos[n + id] = p.y; st.pos[2 * n + id] = p.z;
    }
    if (st.vel) {
        const V4<R> v = vel[w];
        st.vel[id] = v.x; st.vel[n + id] = v.y; st.vel[2 * n + id] = v.z;
    }
    if (st.acc) { st.acc[id] = R(0); st.acc[n + id] = R(0); st.acc[2 * n + id] = R(0); }
    if (st.prs) st.prs[id] = R(0);
    if (st.pav) st.pav[id] = R(0);
    if (st.typ) st.typ[id] = wtyp[w];
}

// per-scene integrals over the listed fluid slots [cs[fbase], cs[fbase + 27 nbxyz])
__device__ __forceinline__ void atomic_max_double(double* a, double v) {
    unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
    unsigned long long old = *p;
    while (__longlong_as_double((long long)old) < v) {
        unsigned long long prev = atomicCAS(p, old, (unsigned long long)__double_as_longlong(v));
        if (prev == old) break;
        old = prev;
    }
}

template <class R, class RN>
__global__ void k_integrals(const SceneDev<R, RN>* scs, const int* cs, const V4<R>* pos,
                            const V4<R>* vel, const int8_t* typ, const int* nbxyz, double* out) {
    const int sidx = blockIdx.y;
    const SceneDev<R, RN>& sc = scs[sidx];
    const int lo = cs[sc.fbase], hi = cs[sc.fbase + 27 * nbxyz[sidx]];
    double cx = 0, cy = 0, cz = 0, ke = 0, fr = -1e300, n = 0;
    for (int s = lo + blockIdx.x * blockDim.x + threadIdx.x; s < hi; s += gridDim.x * blockDim.x) {
        if (typ[s] != kFLD) continue;
        V4<R> p = pos[s], v = vel[s];
        cx += double(p.x); cy += double(p.y); cz += double(p.z);
        ke += 0.5 * (double(v.x) * double(v.x) + double(v.y) * double(v.y) + double(v.z) * double(v.z));
        fr = fmax(fr, double(p.x));
        n += 1;
    }
    for (int o = 16; o > 0; o >>= 1) {
        cx += __shfl_down_sync(0xffffffffu, cx, o);
        cy += __shfl_down_sync(0xffffffffu, cy, o);
        cz += __shfl_down_sync(0xffffffffu, cz, o);
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        n += __shfl_down_sync(0xffffffffu, n, o);
        fr = fmax(fr, __shfl_down_sync(0xffffffffu, fr, o));
    }
    if ((threadIdx.x & 31) == 0) {
        double* o = out + 6 * sidx;
        atomicAdd(o + 0, cx); atomicAdd(o + 1, cy); atomicAdd(o + 2, cz);
        atomicAdd(o + 3, ke); atomicAdd(o + 5, n);
        if (n > 0) atomic_max_double(o + 4, fr);
    }
}

}  // namespace mps
