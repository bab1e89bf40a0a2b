// onBatchCellsOpened on the device (reference MinPlusOracle::onBatchCellsOpened,
// src/minplus_oracle.cpp:530-729, with LeafTile::onBatchCellsOpened,
// src/leaf_tile.cpp:297-374, and InternalNode::applyConwayPerturbations,
// src/internal_node.cpp:332-413) as ONE cooperative persistent kernel.
//
// The host buckets the opened cells (touched leaves with their new in-leaf
// edges, seam edges per lowest common ancestor) and uploads them once.  The
// kernel then walks the levels l = 0..H itself:
//
//   list(l)    leaves: the touched leaves.  Nodes: the nodes holding new
//              seams (placed first by the host) and the parents of every
//              level-(l-1) matrix whose exterior block decreased, appended
//              by the CTA that saw the decrease (a per-node stamp makes each
//              node appear once) - the reference's active parents.
//   insert(l)  leaves: the opened edges (w < D[u][v]: set both entries, mark
//              u and v as pivots).  Nodes: every entry of a decreased child's
//              summary that is smaller than the node's entry (the
//              reference's ChildDecrease list) and the seams.
//   compact(l) pivot flags -> sorted pivot list per matrix.
//   rounds     blocked pivot-set Kleene closure, kOpenB pivots per round:
//              panel: every CTA of a column tile closes the round's pivot
//                block T = D[K, K] itself (Floyd-Warshall in shared memory)
//                and computes P[:, tile] = T* (x) D[K, tile];
//              update: D = min(D, P^T (x) P) over upper-triangle tiles, each
//                also written transposed (D is symmetric), and only where an
//                entry changed.
//              Pipelined one round deep: the panel of round r runs in the
//              same phase as the update of round r - 1 and applies that
//              update to its own pivot rows; round 0's panels run in the
//              compaction's phase, each after its slot's record (R rounds:
//              the compaction phase + R phases).
//   A matrix whose exterior block decreased (refreshBoundarySummary,
//   leaf_tile.cpp:253-273, internal_node.cpp:415-433) is seen where the
//   decrease happens: an insert or an update tile lowers an entry whose row
//   and column are both exterior ports.  No snapshot, no host round trip.
//
// Phases are separated by grid barriers whose waits are bounded: after the
// poll limit a CTA records a timeout in the status word and every CTA
// returns.  Work units inside a phase are handed out by a ticket that the
// barrier resets.  Every sum is the exact clamped tropical product of
// minplus.cuh, and the closure of a matrix over its pivot set is unique, so
// the result equals the reference's bit for bit.
#include "kernels.cuh"
#include "minplus.cuh"

#include <algorithm>

namespace hb {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int B = kOpenB;
constexpr unsigned kBarrierPolls = 1u << 24;
constexpr int kInsertSmem = 64 * 1024;  // staged child rows + node row segments per insert unit

__device__ __forceinline__ unsigned long long global_timer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier ending phase `phase` (0, 1, ... in launch order): every CTA
// adds one to the arrival count L.bar[0] (zero at launch, never reset) and
// waits until it reaches (phase + 1) x grid, so the barrier costs one atomic
// and the polls.  Bounded: a CTA that polls too long records status 1; a CTA
// that sees a non-zero status stops waiting.  Returns false when the launch
// must end.
// Work tickets: phase p hands out units from counter L.bar[1 + p % 2]; CTA i
// takes unit i first without a ticket.  CTA 0 clears the counter of phase
// p + 1 before it arrives at barrier p (its last use was phase p - 1, and
// the barrier publishes the store before phase p + 1 starts).
// s_unit (shared): [0] the unit, [1] -1 until the CTA's first unit of the
// phase is taken, [2] the phase's counter, [3] the CTA's first unit (its
// place in the SM-aware order, sm_order).
__device__ bool open_barrier(const OpenLaunch& L, int phase, int* s_unit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (blockIdx.x == 0) *(volatile unsigned*)(L.bar + 1 + ((phase + 1) & 1)) = 0u;
        __threadfence();
        atomicAdd(L.bar, 1u);
        const unsigned target = (unsigned)(phase + 1) * gridDim.x;
        int ok = 1;
        unsigned it = 0;
        while (ld_acquire(L.bar) < target) {
            if (*(volatile int*)L.status != 0) {
                ok = 0;
                break;
            }
            if (++it > kBarrierPolls) {
                atomicCAS(L.status, 0, 1);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        s_ok = ok && *(volatile int*)L.status == 0;
        s_unit[1] = -1;
        s_unit[2] = (phase + 1) & 1;
    }
    __syncthreads();
    return s_ok != 0;
}

// Next work unit of the phase for this CTA (all threads get it).
__device__ __forceinline__ int next_unit(const OpenLaunch& L, int* s_unit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_unit[1] < 0) {
            s_unit[0] = s_unit[3];
            s_unit[1] = 0;
        } else {
            s_unit[0] = (int)gridDim.x + (int)atomicAdd(L.bar + 1 + s_unit[2], 1u);
        }
    }
    __syncthreads();
    return s_unit[0];
}

// Data that other CTAs of this launch wrote (work lists, slot records,
// stamps, matrices, panels, flags) is read through L2 only (ld.global.cg /
// cp.async.cg): the L1 of this SM may still hold a line of it from before the
// write, and grid barriers do not invalidate L1.
__device__ __forceinline__ int4 ld_slot(const int4* p) { return __ldcg(p); }
__device__ __forceinline__ OpenSlotRec ld_rec(const OpenSlotRec* p) {
    static_assert(sizeof(OpenSlotRec) == 32, "two 16-byte loads");
    const uint4 a = __ldcg(reinterpret_cast<const uint4*>(p));
    const uint4 b = __ldcg(reinterpret_cast<const uint4*>(p) + 1);
    OpenSlotRec r;
    uint4* d = reinterpret_cast<uint4*>(&r);
    d[0] = a;
    d[1] = b;
    return r;
}

__device__ __forceinline__ uint16_t* node_mat(const OpenTaskLevel& T, int node, int NP) {
    return T.mat + (size_t)node * NP * NP;
}

// The exterior block of matrix `node` of level l decreased in this call:
// record it once and list its parent for level l + 1 (once per call).
__device__ void mark_dec(const OpenLaunch& L, int l, int task, int node) {
    const OpenTask& T = L.tasks[task];
    if (l >= T.H) return;  // the root has no summary above it
    if (atomicExch(T.lv[l].dstamp + node, T.stamp) == T.stamp) return;
    const int nx = T.lv[l].nodes_x, g = T.g;
    const int p = ((node / nx) / g) * T.lv[l + 1].nodes_x + (node % nx) / g;
    const int q = ((node / nx) % g) * g + (node % nx) % g;
    {   // the parent's insert phase scans this child's summary
        const int di = atomicAdd(L.dcount + l + 1, 1);
        if (di >= L.cap[l]) {
            atomicCAS(L.status, 0, 2);
            return;
        }
        L.dchild[l + 1][di] = make_int4(task, node, p, q);
    }
    if (atomicExch(T.lv[l + 1].mstamp + p, T.stamp) == T.stamp) return;
    const int idx = atomicAdd(L.count + l + 1, 1);
    if (idx >= L.cap[l + 1]) {
        atomicCAS(L.status, 0, 2);
        return;
    }
    L.slots[l + 1][idx] = make_int4(task, p, 0, 0);
    atomicAdd(&T.out->n_dirty, 1);
}

// ---------------------------------------------------------------------------
// Phase 0: the seam nodes at the head of every level's list are stamped as
// listed, so that a parent appended later is never listed twice.
// ---------------------------------------------------------------------------
__device__ void stamp_phase(const OpenLaunch& L) {
    const int gt = blockIdx.x * kThreads + threadIdx.x, gs = gridDim.x * kThreads;
    // the touched leaves too: an incremental query re-lifts the viewpoints
    // under any listed matrix (htrip_query_all_pairs_incremental)
    const int n0 = min(*(volatile int*)L.count, L.cap[0]);
    for (int s = gt; s < n0; s += gs) {
        const int4 e = L.slots[0][s];
        const OpenTask& T = L.tasks[e.x];
        T.lv[0].mstamp[e.y] = T.stamp;
    }
    for (int l = 1; l <= L.maxH; ++l)
        for (int s = gt; s < L.n_seam[l]; s += gs) {
            const int4 e = ld_slot(L.slots[l] + s);
            const OpenTask& T = L.tasks[e.x];
            T.lv[l].mstamp[e.y] = T.stamp;
        }
}

// ---------------------------------------------------------------------------
// Insert phase.
// ---------------------------------------------------------------------------
// Edge / seam list of one slot (leaf_tile.cpp:311-330,
// internal_node.cpp:356-365), one warp: an entry counts, and its endpoints
// become pivots, only if it shortens D[u][v].  The lanes take the entries in
// parallel: a pair listed twice (both cells opened) has the same weight, so
// the set of shortened pairs, and the pivots, are those of the sequential
// loop; a pivot flag counts once (atomicOr on its 4-byte word).
__device__ void insert_list(const OpenLaunch& L, int l, int4 e, int* new_pivots, bool* dec) {
    const OpenTask& T = L.tasks[e.x];
    const OpenLevelGeom& G = L.geo[l];
    const int NP = G.NP, lane = threadIdx.x & 31;
    uint16_t* D = node_mat(T.lv[l], e.y, NP);
    uint8_t* f = T.lv[l].kflag + (size_t)e.y * NP;
    int np = 0;
    bool d = false;
    for (int t = e.z + lane; t < e.w; t += 32) {
        const int u = L.triples[3 * t], v = L.triples[3 * t + 1];
        const uint16_t w = (uint16_t)L.triples[3 * t + 2];
        if (w < __ldcg(D + (size_t)u * NP + v)) {
            D[(size_t)u * NP + v] = w;
            D[(size_t)v * NP + u] = w;
            const int ends[2] = {u, v};
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                const int a = ends[x];
                const unsigned sh = (unsigned)(a & 3) * 8u;
                const unsigned old = atomicOr(reinterpret_cast<unsigned*>(f + (a & ~3)), 1u << sh);
                np += ((old >> sh) & 0xffu) == 0;
            }
            d |= G.isext[u] && G.isext[v];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) np += __shfl_xor_sync(FULL, np, o);
    *new_pivots = np;
    *dec = __any_sync(FULL, d);
}

// Rows of a decreased child's summary an insert unit takes: the child rows
// and the node's row segments of the block staged in shared memory fit
// kInsertSmem bytes; 0 when one row does not fit (a unit then takes one row
// and reads it from global memory).
__device__ __forceinline__ int insert_rows(const OpenLevelGeom& G) {
    const int seg = ((G.nP + 7) / 8 + 1) * 8;  // the node's row segment, 16-byte aligned, rounded out
    const int per_row = (G.childNP + seg) * (int)sizeof(uint16_t);
    return min(G.nP, (int)(kInsertSmem / per_row));
}

// Insert phase of level l.  Units: the slots' edge / seam lists (one warp
// per slot), then, for levels >= 1, every child whose summary decreased in
// this call (listed by mark_dec) in blocks of at most insert_rows(G) rows of its
// nP x nP summary: every summary entry smaller than the node's entry is
// inserted (internal_node.cpp:343-353) - the same as inserting the
// reference's decrease list, since an entry that did not decrease is never
// smaller than the node's, which is <= the old summary.  A unit stages the
// whole child rows and the node's row segments in shared memory with
// asynchronous 16-byte copies (one round trip), then compares there.
__device__ void insert_phase(const OpenLaunch& L, int l, int N, int* s_unit, unsigned char* smem) {
    const OpenLevelGeom& G = L.geo[l];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ int s_dec;
    const int list_units = (N + kWarps - 1) / kWarps;
    const int nd = l >= 1 ? min(*(volatile int*)(L.dcount + l), L.cap[l - 1]) : 0;
    const int R0 = l >= 1 ? insert_rows(G) : 1;
    const bool staged = R0 > 0;
    // about two row blocks per CTA over the level's decreased children,
    // within what shared memory holds
    const int R = staged ? max(1, min(R0, (G.nP * nd + 2 * (int)gridDim.x - 1) / (2 * (int)gridDim.x))) : 1;
    const int blocks = l >= 1 ? (G.nP + R - 1) / R : 0;
    const int units = list_units + nd * blocks;
    for (int u = next_unit(L, s_unit); u < units; u = next_unit(L, s_unit)) {
        if (u < list_units) {
            const int s = u * kWarps + warp;
            if (s < N) {
                const int4 e = ld_slot(L.slots[l] + s);
                if (e.w > e.z) {  // uniform over the warp
                    int np = 0;
                    bool dec = false;
                    insert_list(L, l, e, &np, &dec);
                    if (lane == 0) {
                        const OpenTask& T = L.tasks[e.x];
                        if (l == 0 && np) atomicAdd(&T.out->new_pivots, np);
                        if (dec) mark_dec(L, l, e.x, e.y);
                    }
                }
            }
            continue;
        }
        const int cu = u - list_units;
        const int4 dc = ld_slot(L.dchild[l] + cu / blocks);  // {task, child, node, quad}
        const OpenTask& T = L.tasks[dc.x];
        const int NP = G.NP, nP = G.nP, cNP = G.childNP, q = dc.w;
        const int p0 = (cu % blocks) * R, rows = min(R, nP - p0);
        const int col0 = q * nP, c_lo = col0 & ~7;
        const int seg = ((nP + 7) / 8 + 1) * 8;  // covers [c_lo, col0 + nP)
        const uint16_t* cm = node_mat(T.lv[l - 1], dc.y, cNP);
        uint16_t* D = node_mat(T.lv[l], dc.z, NP);
        uint8_t* f = T.lv[l].kflag + (size_t)dc.z * NP;
        uint16_t* Cs = reinterpret_cast<uint16_t*>(smem);  // [rows][cNP] child rows
        uint16_t* Ps = Cs + (size_t)rows * cNP;            // [rows][seg] node row segments
        if (threadIdx.x == 0) s_dec = 0;
        bool dec = false;
        if (!staged) {  // one row straight from global memory
            __syncthreads();
            const int ra = col0 + p0;
            const uint16_t* crow = cm + (size_t)G.child_ext[p0] * cNP;
            for (int pp = threadIdx.x; pp < nP; pp += kThreads) {
                const int cb = col0 + pp;
                const uint16_t w = __ldcg(crow + G.child_ext[pp]);
                if (w < __ldcg(D + (size_t)ra * NP + cb)) {
                    D[(size_t)ra * NP + cb] = w;  // (cb, ra) is written by the unit of row cb
                    f[ra] = 1;
                    f[cb] = 1;
                    dec |= G.isext[ra] && G.isext[cb];
                }
            }
        } else {
            for (int idx = threadIdx.x; idx < rows * (cNP / 8); idx += kThreads) {
                const int r = idx / (cNP / 8), c8 = idx - r * (cNP / 8);
                cp_async16(Cs + (size_t)r * cNP + c8 * 8, cm + (size_t)G.child_ext[p0 + r] * cNP + c8 * 8);
            }
            for (int idx = threadIdx.x; idx < rows * (seg / 8); idx += kThreads) {
                const int r = idx / (seg / 8), c8 = idx - r * (seg / 8);
                // the segment's last chunk may reach past the row (into the
                // next row, or past the matrix): only [col0, col0 + nP) is used
                const size_t off = (size_t)(col0 + p0 + r) * NP + c_lo + c8 * 8;
                if (off + 8 <= (size_t)NP * NP) cp_async16(Ps + r * seg + c8 * 8, D + off);
            }
            cp_async_wait_all();
            __syncthreads();
            int r = threadIdx.x / nP, pp = threadIdx.x - r * nP;  // entry (r, pp) = r nP + pp, walked
            for (int idx = threadIdx.x; idx < rows * nP; idx += kThreads) {
                const uint16_t w = Cs[(size_t)r * cNP + G.child_ext[pp]];
                if (w < Ps[r * seg + (col0 - c_lo) + pp]) {
                    const int ra = col0 + p0 + r, cb = col0 + pp;
                    D[(size_t)ra * NP + cb] = w;  // (cb, ra) is written by the unit of row cb
                    f[ra] = 1;
                    f[cb] = 1;
                    dec |= G.isext[ra] && G.isext[cb];
                }
                pp += kThreads;
                while (pp >= nP) {
                    pp -= nP;
                    ++r;
                }
            }
        }
        if (__any_sync(FULL, dec) && lane == 0) s_dec = 1;
        __syncthreads();
        if (threadIdx.x == 0 && s_dec) mark_dec(L, l, dc.x, dc.z);
    }
}

// ---------------------------------------------------------------------------
// Compaction (one unit per slot): the pivot flags become the ascending pivot
// list (and are cleared); per-level statistics and the largest pivot count
// of the level (which sets the number of rounds); the slot's record, then
// its ready flag.
// ---------------------------------------------------------------------------
__device__ void compact_unit(const OpenLaunch& L, int l, int s) {
    const OpenLevelGeom& G = L.geo[l];
    __shared__ int warp_tot[kWarps];
    __shared__ int base;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    {
        const int4 e = ld_slot(L.slots[l] + s);
        const OpenTask& T = L.tasks[e.x];
        uint8_t* f = T.lv[l].kflag + (size_t)e.y * G.NP;
        int* out = T.lv[l].klist + (size_t)e.y * G.NP;
        if (threadIdx.x == 0) base = 0;
        __syncthreads();
        // each thread takes 4 consecutive flags (one 32-bit word) per step
        for (int j0 = 0; j0 < G.NP; j0 += 4 * kThreads) {
            const int j = j0 + 4 * threadIdx.x;
            unsigned wv = 0;
            if (j < G.NP) wv = __ldcg(reinterpret_cast<const unsigned*>(f + j));
            const int cnt = (wv & 0xffu ? 1 : 0) + (wv & 0xff00u ? 1 : 0) + (wv & 0xff0000u ? 1 : 0) +
                            (wv & 0xff000000u ? 1 : 0);
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            if (lane == 31) warp_tot[warp] = incl;
            __syncthreads();
            int off = base + incl - cnt;
            for (int w = 0; w < warp; ++w) off += warp_tot[w];
            if (wv) {
#pragma unroll
                for (int x = 0; x < 4; ++x)
                    if ((wv >> (8 * x)) & 0xffu) out[off++] = j + x;
                *reinterpret_cast<unsigned*>(f + j) = 0u;
            }
            __syncthreads();
            if (threadIdx.x == 0)
                for (int w = 0; w < kWarps; ++w) base += warp_tot[w];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const int k = base;
            T.lv[l].kcnt[e.y] = k;
            L.rec[l][s] = OpenSlotRec{node_mat(T.lv[l], e.y, G.NP), out, k, e.x, e.y, 0};
            __threadfence();  // the pivot list and the record, then the release
            atomicExch(&L.rec[l][s].ready, 1);
            atomicAdd(&T.out->level[l][0], 1);
            atomicAdd(&T.out->level[l][1], k);
            atomicMax(&T.out->level[l][2], k);
            atomicMax(L.maxk + l, k);
            if (k) {
                const unsigned long long n = (unsigned long long)G.n;
                atomicAdd(&T.out->ops, n * n * (unsigned long long)k);
                atomicAdd(&T.out->bytes, 4ull * n * n + 4ull * (unsigned long long)k * n);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Panel unit of round r: (slot, column tile of 64 columns).
//   T* = closure of T = D[Kc, Kc] (Floyd-Warshall over the round's pivots, in
//        shared memory; the reference's sequential relaxation restricted to
//        the pivots),
//   P[a][j] = min_c T*[a][c] (+) D[Kc[c]][j]   for the tile's columns j,
// both from one Floyd-Warshall pass over the pivot rows [T | D[Kc, tile]],
// stored in the slot's panel, with the 64-column blocks holding a finite
// value flagged for the update.
// ---------------------------------------------------------------------------
constexpr int kTLD = B + 8;  // padded row of T (144 bytes): column reads hit distinct banks

// Floyd-Warshall over the round's pivot block T (mk <= B rows, identity
// beyond) in shared memory: thread t owns row t / 4 and 16 columns.  Step kk
// reads row kk and column kk, whose values it rewrites unchanged
// (T[kk][kk] = 0), so one barrier per step orders it before step kk + 1; a
// = INF gives no change through the clamped form, so no branch is needed.
__device__ __forceinline__ void close_pivot_block(uint16_t (*Ts)[kTLD], int mk) {
    const int tid = threadIdx.x;
    const int a = tid >> 2, c0 = (tid & 3) * 16;
    uint32_t v[8];
    const uint4 x0 = *reinterpret_cast<const uint4*>(&Ts[a][c0]);
    const uint4 y0 = *reinterpret_cast<const uint4*>(&Ts[a][c0 + 8]);
    v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w; v[4] = y0.x; v[5] = y0.y; v[6] = y0.z; v[7] = y0.w;
    for (int kk = 0; kk < mk; ++kk) {
        const uint32_t t = Ts[a][kk];
        const uint4 x = *reinterpret_cast<const uint4*>(&Ts[kk][c0]);
        const uint4 y = *reinterpret_cast<const uint4*>(&Ts[kk][c0 + 8]);
        const uint32_t rw[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
        const uint32_t aa = splat(t), tt = INF2 - aa;
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = acc_clamp(v[i], rw[i], aa, tt);
        *reinterpret_cast<uint4*>(&Ts[a][c0]) = make_uint4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<uint4*>(&Ts[a][c0 + 8]) = make_uint4(v[4], v[5], v[6], v[7]);
        __syncthreads();
    }
}

// Floyd-Warshall over the round's pivots on the augmented rows [T | Bt]:
// T the pivot block as above, Bt the pivot rows of a 64-column tile.  After
// the last pivot, Bt = T* (x) Bt: a shortest path from pivot a to column j
// through pivots ends with one entry D[c][j] of a pivot row.  Thread t owns
// row t / 4 and 16 columns of each part; its Bt values end in vb.  Row kk of
// both parts is rewritten unchanged at step kk (T[kk][kk] = 0), so one
// barrier per step; rows >= mk of Bt are never read (T[a][kk] = INF there).
__device__ __forceinline__ void close_pivot_panel(uint16_t (*Ts)[kTLD], uint16_t (*Bt)[kTLD], int mk,
                                                  uint32_t (&vb)[8]) {
    const int tid = threadIdx.x;
    const int a = tid >> 2, c0 = (tid & 3) * 16;
    uint32_t v[8];
    {
        const uint4 x0 = *reinterpret_cast<const uint4*>(&Ts[a][c0]);
        const uint4 y0 = *reinterpret_cast<const uint4*>(&Ts[a][c0 + 8]);
        const uint4 x1 = *reinterpret_cast<const uint4*>(&Bt[a][c0]);
        const uint4 y1 = *reinterpret_cast<const uint4*>(&Bt[a][c0 + 8]);
        v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w; v[4] = y0.x; v[5] = y0.y; v[6] = y0.z; v[7] = y0.w;
        vb[0] = x1.x; vb[1] = x1.y; vb[2] = x1.z; vb[3] = x1.w; vb[4] = y1.x; vb[5] = y1.y; vb[6] = y1.z; vb[7] = y1.w;
    }
    for (int kk = 0; kk < mk; ++kk) {
        const uint32_t t = Ts[a][kk];
        const uint4 x = *reinterpret_cast<const uint4*>(&Ts[kk][c0]);
        const uint4 y = *reinterpret_cast<const uint4*>(&Ts[kk][c0 + 8]);
        const uint4 xb = *reinterpret_cast<const uint4*>(&Bt[kk][c0]);
        const uint4 yb = *reinterpret_cast<const uint4*>(&Bt[kk][c0 + 8]);
        const uint32_t rw[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
        const uint32_t rb[8] = {xb.x, xb.y, xb.z, xb.w, yb.x, yb.y, yb.z, yb.w};
        const uint32_t aa = splat(t), tt = INF2 - aa;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            v[i] = acc_clamp(v[i], rw[i], aa, tt);
            vb[i] = acc_clamp(vb[i], rb[i], aa, tt);
        }
        *reinterpret_cast<uint4*>(&Ts[a][c0]) = make_uint4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<uint4*>(&Ts[a][c0 + 8]) = make_uint4(v[4], v[5], v[6], v[7]);
        *reinterpret_cast<uint4*>(&Bt[a][c0]) = make_uint4(vb[0], vb[1], vb[2], vb[3]);
        *reinterpret_cast<uint4*>(&Bt[a][c0 + 8]) = make_uint4(vb[4], vb[5], vb[6], vb[7]);
        __syncthreads();
    }
}

// Class of pivot k for warp w's 8 rows of T* (entries T*[k][8w .. 8w+7]):
// 0 all INF (skip), 1 all <= INF_HEADROOM (2-op form), 2 otherwise.
__device__ __forceinline__ void panel_classes(uint16_t (*Ts)[kTLD], int mk, uint8_t* cls) {
    for (int idx = threadIdx.x; idx < mk * kWarps; idx += kThreads) {
        const int k = idx / kWarps, w = idx % kWarps;
        uint32_t mn = 0xffffu, mx = 0;
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
            const uint32_t v = Ts[k][w * 8 + rr];
            mn = min(mn, v);
            mx = max(mx, v);
        }
        cls[idx] = mn >= INF ? 0 : (mx <= INF_HEADROOM ? 1 : 2);
    }
}

// acc[r][c] = min_k T*[k][8w + r] (+) Bs[k][lane's pair c]  (T* symmetric:
// T*[k][a] = T*[a][k]); warp w owns pivot rows 8w..8w+7.
template <int CP>
__device__ __forceinline__ void panel_gemm(uint16_t (*Ts)[kTLD], const uint16_t* Bs, int ldb, int mk,
                                           const uint8_t* cls, uint32_t (&acc)[8][CP]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int rr = 0; rr < 8; ++rr)
#pragma unroll
        for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = INF2;
    if constexpr (CP == 1) {
        // one column pair per lane: little work per pivot, so the loop is
        // latency-bound; it runs branch-free (the clamped form is exact for
        // every value, INF included) and unrolled, so the shared-memory loads
        // of later pivots overlap the arithmetic of earlier ones
        (void)cls;
#pragma unroll 4
        for (int k = 0; k < mk; ++k) {
            const uint32_t bv = reinterpret_cast<const uint32_t*>(Bs + k * ldb + lane * 2)[0];
            const uint4 av = *reinterpret_cast<const uint4*>(&Ts[k][warp * 8]);
            const uint32_t aw[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
            for (int r2 = 0; r2 < 4; ++r2) {
                const uint32_t a0 = splat(aw[r2]), a1 = splat(aw[r2] >> 16);
                acc[2 * r2][0] = acc_clamp(acc[2 * r2][0], bv, a0, INF2 - a0);
                acc[2 * r2 + 1][0] = acc_clamp(acc[2 * r2 + 1][0], bv, a1, INF2 - a1);
            }
        }
    } else {
        for (int k = 0; k < mk; ++k) {
            const int c = cls[k * kWarps + warp];
            if (c == 0) continue;  // uniform over the warp
            uint32_t bv[CP];
#pragma unroll
            for (int cc = 0; cc < CP; ++cc) bv[cc] = reinterpret_cast<const uint32_t*>(Bs + k * ldb + lane * 2 * CP)[cc];
            const uint4 av = *reinterpret_cast<const uint4*>(&Ts[k][warp * 8]);
            const uint32_t aw[4] = {av.x, av.y, av.z, av.w};
            uint32_t aa[8];
#pragma unroll
            for (int r2 = 0; r2 < 4; ++r2) {
                aa[2 * r2] = splat(aw[r2]);
                aa[2 * r2 + 1] = splat(aw[r2] >> 16);
            }
            if (c == 1) {
#pragma unroll
                for (int rr = 0; rr < 8; ++rr)
#pragma unroll
                    for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = acc_fast(acc[rr][cc], bv[cc], aa[rr]);
            } else {
#pragma unroll
                for (int rr = 0; rr < 8; ++rr) {
                    const uint32_t tt = INF2 - aa[rr];
#pragma unroll
                    for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = acc_clamp(acc[rr][cc], bv[cc], aa[rr], tt);
                }
            }
        }
    }
}

__device__ __forceinline__ uint16_t* panel_of(const OpenLaunch& L, int r, int s, int NP) {
    return L.panel + (size_t)(r & 1) * L.panel_stride + (size_t)s * B * NP;
}
__device__ __forceinline__ uint8_t* pflags_of(const OpenLaunch& L, int r, int s, int NP) {
    return L.pflags + (size_t)(r & 1) * L.pflag_stride + (size_t)s * (NP / 64);
}

// 64 x 64 block product of the panel unit (kn <= B pivot steps):
//   acc[i][q] = min_k A[k][row i] (+) Bm[k][column pair q]
// Warp w owns rows 8w .. 8w + 7 and skips (class 0) or takes the 2-op form
// (class 1) for pivot k by cls[k * kWarps + w]; lane 8 rp + cg holds rows
// 8w + 2rp, 8w + 2rp + 1 and columns 8cg .. 8cg + 7 (four packed pairs), so
// a pivot step is one 4-byte and one 16-byte shared load for 8 updates.
__device__ __forceinline__ void gemm64(const uint16_t (*A)[kTLD], const uint16_t* Bm, int ldb, int kn,
                                       const uint8_t* cls, uint32_t (&acc)[2][4]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint16_t* ap = &A[0][warp * 8 + 2 * (lane >> 3)];
    const uint16_t* bp = Bm + (lane & 7) * 8;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = INF2;
#pragma unroll 2
    for (int k = 0; k < kn; ++k) {
        const int c = cls[k * kWarps + warp];
        if (c == 0) continue;  // uniform over the warp
        const uint32_t a2 = *reinterpret_cast<const uint32_t*>(ap + k * kTLD);
        const uint4 b4 = *reinterpret_cast<const uint4*>(bp + k * ldb);
        const uint32_t b[4] = {b4.x, b4.y, b4.z, b4.w};
        const uint32_t aa[2] = {splat(a2), splat(a2 >> 16)};
        if (c == 1) {
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[i][q] = acc_fast(acc[i][q], b[q], aa[i]);
        } else {
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const uint32_t tt = INF2 - aa[i];
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[i][q] = acc_clamp(acc[i][q], b[q], aa[i], tt);
            }
        }
    }
}

// dst[row i][8 cg .. 8 cg + 7] = min(dst, acc[i]) for the rows of gemm64's
// thread layout below `rows`.
__device__ __forceinline__ void min_into(uint16_t* dst, int ld, int rows, const uint32_t (&acc)[2][4]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int a = warp * 8 + 2 * (lane >> 3) + i;
        if (a >= rows) continue;
        uint4* p = reinterpret_cast<uint4*>(dst + a * ld + (lane & 7) * 8);
        const uint4 o = *p;
        *p = make_uint4(min2(o.x, acc[i][0]), min2(o.y, acc[i][1]), min2(o.z, acc[i][2]), min2(o.w, acc[i][3]));
    }
}

// Class of step k for warp w's rows of a 64 x 64 operand A (entries
// A[k][8w .. 8w+7]): 0 all INF (skip), 1 all <= INF_HEADROOM (2-op form),
// 2 otherwise.
__device__ __forceinline__ void block_classes(const uint16_t (*A)[kTLD], int kn, uint8_t* cls) {
    for (int idx = threadIdx.x; idx < kn * kWarps; idx += kThreads) {
        const int k = idx / kWarps, w = idx % kWarps;
        const uint4 v = *reinterpret_cast<const uint4*>(&A[k][w * 8]);
        const uint32_t x[4] = {v.x, v.y, v.z, v.w};
        uint32_t mn = 0xffffu, mx = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            mn = min(mn, min(x[q] & 0xffffu, x[q] >> 16));
            mx = max(mx, max(x[q] & 0xffffu, x[q] >> 16));
        }
        cls[idx] = mn >= INF ? 0 : (mx <= INF_HEADROOM ? 1 : 2);
    }
}

// Panel unit of round r >= 1 runs beside the update of round r - 1 (the
// look-ahead): the pivot rows D[Kc, :] it reads may not hold that update
// yet, so it applies it itself from round r - 1's panel Pp (all of its
// B rows in use: only the last round of a slot has fewer pivots),
//   D[Kc[a]][j] = min(D[Kc[a]][j], min_c Pp[c][Kc[a]] (+) Pp[c][j]),
// to the pivot block and to the tile's columns.  A value it reads either
// still misses the update or already holds it; the minimum is the updated
// value both ways, so the panel equals the one made after the update.
__device__ void panel_unit(const OpenLaunch& L, int l, int s, int j0, int r, unsigned char* smem) {
    constexpr int NT = 64;
    const int NP = L.geo[l].NP;
    const OpenSlotRec rec = ld_rec(L.rec[l] + s);
    const int mk = min(B, rec.kcnt - r * B);
    if (mk <= 0) return;  // uniform
    const bool ahead = r > 0;
    uint16_t (*Ts)[kTLD] = reinterpret_cast<uint16_t (*)[kTLD]>(smem);
    uint16_t (*Ag)[kTLD] = reinterpret_cast<uint16_t (*)[kTLD]>(smem + B * kTLD * sizeof(uint16_t));  // Pp[c][Kc[a]]
    uint16_t (*Bt)[kTLD] = reinterpret_cast<uint16_t (*)[kTLD]>(smem + 2 * B * kTLD * sizeof(uint16_t));  // tile rows
    uint16_t* Bs = &Bt[0][0];
    uint16_t* Pj = Bs + B * kTLD;  // [B][NT]: Pp[c][j0 + j]
    int* kc = reinterpret_cast<int*>(Pj + B * NT);
    uint8_t* clsA = reinterpret_cast<uint8_t*>(kc + B);  // [B][kWarps] of Ag
    __shared__ int tile_any;
    const uint16_t* D = rec.mat;
    const uint16_t* Pp = ahead ? panel_of(L, r - 1, s, NP) : nullptr;
    const int tid = threadIdx.x;
    if (tid < mk) kc[tid] = __ldcg(rec.klist + r * B + tid);
    if (tid == 0) tile_any = 0;
    __syncthreads();
    {   // the tile's pivot rows (and round r - 1's panel tile) by asynchronous
        // copies, waited for only where they are used; meanwhile the
        // scattered pivot block (and its round r - 1 panel columns) with
        // all of a thread's loads issued first
        for (int idx = tid; idx < mk * (NT / 8); idx += kThreads) {
            const int a = idx / (NT / 8), c8 = idx % (NT / 8);
            cp_async16(Bs + a * kTLD + c8 * 8, D + (size_t)kc[a] * NP + j0 + c8 * 8);
        }
        if (ahead)
            for (int idx = tid; idx < B * (NT / 8); idx += kThreads) {
                const int c = idx / (NT / 8), c8 = idx % (NT / 8);
                cp_async16(Pj + c * NT + c8 * 8, Pp + (size_t)c * NP + j0 + c8 * 8);
            }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        constexpr int NTB = B * B / kThreads;
        uint16_t tv[NTB], pv[NTB];
#pragma unroll
        for (int x = 0; x < NTB; ++x) {
            const int idx = tid + x * kThreads, a = idx / B, c = idx % B;
            tv[x] = (a < mk && c < mk) ? __ldcg(D + (size_t)kc[a] * NP + kc[c]) : (a == c ? 0 : INF);
            // pv: Pp[a][Kc[c]] (row a of the old panel at pivot c)
            pv[x] = (ahead && c < mk) ? __ldcg(Pp + (size_t)a * NP + kc[c]) : INF;
        }
#pragma unroll
        for (int x = 0; x < NTB; ++x) {
            const int idx = tid + x * kThreads;
            Ts[idx / B][idx % B] = tv[x];
            Ag[idx / B][idx % B] = pv[x];
        }
    }
    __syncthreads();
    uint32_t acc[2][4];
    if (ahead) {  // round r - 1's update of the pivot rows: the pivot block, then the tile's columns
        block_classes(Ag, B, clsA);
        __syncthreads();
        gemm64(Ag, &Ag[0][0], kTLD, B, clsA, acc);
        min_into(&Ts[0][0], kTLD, B, acc);  // rows / columns >= mk: INF from Ag, the identity stays
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
        gemm64(Ag, Pj, NT, B, clsA, acc);
        min_into(Bs, kTLD, mk, acc);
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    uint32_t vb[8];
    close_pivot_panel(Ts, Bt, mk, vb);
    uint16_t* P = panel_of(L, r, s, NP);
    const int lane = tid & 31, a = tid >> 2, c0 = (tid & 3) * 16;
    bool any = false;
    if (a < mk) {
        uint4* dst = reinterpret_cast<uint4*>(P + (size_t)a * NP + j0 + c0);
        dst[0] = make_uint4(vb[0], vb[1], vb[2], vb[3]);
        dst[1] = make_uint4(vb[4], vb[5], vb[6], vb[7]);
#pragma unroll
        for (int i = 0; i < 8; ++i) any |= vb[i] != INF2;
    }
    if (__any_sync(FULL, any) && lane == 0) tile_any = 1;
    __syncthreads();
    if (tid == 0) pflags_of(L, r, s, NP)[j0 / 64] = tile_any ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Update phase of round r: unit = (slot, tile pair I <= J) of TT x TT tiles.
//   D[i][j] = min(D[i][j], min_a P[a][i] (+) P[a][j])   (a < mk)
// computed once for the upper-triangle tile and written to (I, J) and,
// transposed, to (J, I); tiles whose rows or columns hold no finite panel
// value are skipped, unchanged rows are not written.  An exterior x exterior
// entry that decreased marks the matrix's summary as decreased.
// Warp w owns rows RW*w .. RW*w + RW - 1 of the tile, each lane CP column
// pairs.  Per pivot k the warp's RW panel values share one class, staged
// with the panel: 0 all INF (skip), 1 all <= INF_HEADROOM (2-op form, no
// wrap), 2 otherwise (3-op clamped form).
// ---------------------------------------------------------------------------
template <int RW, int CP>
__device__ void update_unit(const OpenLaunch& L, int l, int s, int I, int J, int r, unsigned char* smem) {
    constexpr int TT = 8 * RW;  // == 64 * CP
    static_assert(TT == 64 * CP, "square tiles");
    const OpenLevelGeom& G = L.geo[l];
    const int NP = G.NP;
    const uint8_t* pf = pflags_of(L, r, s, NP);
    const OpenSlotRec rec = ld_rec(L.rec[l] + s);
    const int mk = min(B, rec.kcnt - r * B);
    if (mk <= 0) return;  // uniform; no panel was made for this slot either
    bool live_i = false, live_j = false;
#pragma unroll
    for (int t = 0; t < TT / 64; ++t) {
        live_i |= __ldcg(pf + I * (TT / 64) + t) != 0;
        live_j |= __ldcg(pf + J * (TT / 64) + t) != 0;
    }
    if (!live_i || !live_j) return;  // uniform
    uint32_t* As = reinterpret_cast<uint32_t*>(smem);                                  // [B][TT] splatted
    uint16_t* Bs = reinterpret_cast<uint16_t*>(smem + (size_t)B * TT * sizeof(uint32_t));  // [B][TT]
    uint8_t* cls = smem + (size_t)B * TT * (sizeof(uint32_t) + sizeof(uint16_t));          // [B][kWarps]
    uint16_t* Os = reinterpret_cast<uint16_t*>(cls + B * kWarps);                          // [TT][TT] old tile
    __shared__ int s_any, s_dec;
    const uint16_t* P = panel_of(L, r, s, NP);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i0 = I * TT, jb = J * TT;
    if (tid == 0) { s_any = 0; s_dec = 0; }
    uint16_t* D = rec.mat;
    {   // asynchronous copies of the column panel and of the old tile (read
        // only in the epilogue); the row panel is splatted through registers
        for (int idx = tid; idx < mk * (TT / 8); idx += kThreads) {
            const int a = idx / (TT / 8), c8 = idx % (TT / 8);
            cp_async16(Bs + a * TT + c8 * 8, P + (size_t)a * NP + jb + c8 * 8);
        }
        for (int idx = tid; idx < TT * (TT / 8); idx += kThreads) {
            const int rr = idx / (TT / 8), c8 = idx % (TT / 8);
            cp_async16(Os + rr * TT + c8 * 8, D + (size_t)(i0 + rr) * NP + jb + c8 * 8);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        constexpr int NS = B * (TT / 8) / kThreads;
        uint4 va[NS];
#pragma unroll
        for (int x = 0; x < NS; ++x) {
            const int idx = tid + x * kThreads, a = idx / (TT / 8), c8 = idx % (TT / 8);
            if (a < mk) va[x] = __ldcg(reinterpret_cast<const uint4*>(P + (size_t)a * NP + i0) + c8);
        }
#pragma unroll
        for (int x = 0; x < NS; ++x) {
            const int idx = tid + x * kThreads, a = idx / (TT / 8), c8 = idx % (TT / 8);
            if (a < mk) {
                const uint32_t w[4] = {va[x].x, va[x].y, va[x].z, va[x].w};
                uint4* dst = reinterpret_cast<uint4*>(As + a * TT + c8 * 8);
                dst[0] = make_uint4(splat(w[0]), splat(w[0] >> 16), splat(w[1]), splat(w[1] >> 16));
                dst[1] = make_uint4(splat(w[2]), splat(w[2] >> 16), splat(w[3]), splat(w[3] >> 16));
            }
        }
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    for (int idx = tid; idx < mk * kWarps; idx += kThreads) {
        const int a = idx / kWarps, w = idx % kWarps;
        const uint32_t* ar = As + a * TT + w * RW;
        uint32_t mn = 0xffffu, mx = 0;
#pragma unroll
        for (int rr = 0; rr < RW; ++rr) {
            const uint32_t v = ar[rr] & 0xffffu;
            mn = min(mn, v);
            mx = max(mx, v);
        }
        cls[idx] = mn >= INF ? 0 : (mx <= INF_HEADROOM ? 1 : 2);
    }
    __syncthreads();
    uint32_t acc[RW][CP];
#pragma unroll
    for (int rr = 0; rr < RW; ++rr)
#pragma unroll
        for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = INF2;
    for (int k = 0; k < mk; ++k) {
        const int c = cls[k * kWarps + warp];
        if (c == 0) continue;  // uniform over the warp
        uint32_t bv[CP];
#pragma unroll
        for (int cc = 0; cc < CP; ++cc) bv[cc] = reinterpret_cast<const uint32_t*>(Bs + k * TT + lane * 2 * CP)[cc];
        const uint32_t* ar = As + k * TT + warp * RW;
        uint32_t av[RW];
#pragma unroll
        for (int q = 0; q < RW / 4; ++q) {
            const uint4 x = reinterpret_cast<const uint4*>(ar)[q];
            av[4 * q] = x.x; av[4 * q + 1] = x.y; av[4 * q + 2] = x.z; av[4 * q + 3] = x.w;
        }
        if (c == 1) {
#pragma unroll
            for (int rr = 0; rr < RW; ++rr)
#pragma unroll
                for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = acc_fast(acc[rr][cc], bv[cc], av[rr]);
        } else {
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                const uint32_t tt = INF2 - av[rr];
#pragma unroll
                for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = acc_clamp(acc[rr][cc], bv[cc], av[rr], tt);
            }
        }
    }
    // epilogue: new = min(acc, old); changed entries are written
    const int col = jb + lane * 2 * CP;
    uint32_t cext[CP];
#pragma unroll
    for (int cc = 0; cc < CP; ++cc)
        cext[cc] = (G.isext[col + 2 * cc] ? 0xffffu : 0u) | (G.isext[col + 2 * cc + 1] ? 0xffff0000u : 0u);
    bool any = false, dec = false;
#pragma unroll
    for (int rr = 0; rr < RW; ++rr) {
        const int row = i0 + warp * RW + rr;
        uint32_t* dp = reinterpret_cast<uint32_t*>(D + (size_t)row * NP + col);
        const bool rext = G.isext[row] != 0;
        const uint32_t* old = reinterpret_cast<const uint32_t*>(Os + (warp * RW + rr) * TT + lane * 2 * CP);
        uint32_t ch = 0;
#pragma unroll
        for (int cc = 0; cc < CP; ++cc) {
            acc[rr][cc] = min2(acc[rr][cc], old[cc]);
            const uint32_t diff = acc[rr][cc] ^ old[cc];
            ch |= diff;
            if (rext) dec |= (diff & cext[cc]) != 0;
        }
        if (ch) {
            any = true;
            if constexpr (CP == 2) {
                *reinterpret_cast<uint2*>(dp) = make_uint2(acc[rr][0], acc[rr][1]);  // one 8-byte store
            } else {
#pragma unroll
                for (int cc = 0; cc < CP; ++cc) dp[cc] = acc[rr][cc];
            }
        }
    }
    if (__any_sync(FULL, any) && lane == 0) s_any = 1;
    if (__any_sync(FULL, dec) && lane == 0) s_dec = 1;
    __syncthreads();  // the staging buffers are free from here on
    if (I != J && s_any) {
        // The transposed tile through shared memory, Tt[j][i] in 16-byte
        // chunks of 8 rows i: a thread holds RW consecutive rows of each of
        // its columns, i.e. whole chunks of a transposed row.  Chunk q of row
        // j sits at q ^ ((j / (2 CP)) & 7), so the 8 lanes of a 16-byte store
        // phase (8 different rows) hit 8 different bank groups.
        uint16_t* Tt = reinterpret_cast<uint16_t*>(smem);
#pragma unroll
        for (int cc = 0; cc < CP; ++cc)
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                const int j = lane * 2 * CP + 2 * cc + x;
                const int key = (j / (2 * CP)) & 7;
#pragma unroll
                for (int h = 0; h < RW / 8; ++h) {
                    uint32_t w4[4];
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const uint32_t a = x ? (acc[8 * h + 2 * t][cc] >> 16) : (acc[8 * h + 2 * t][cc] & 0xffffu);
                        const uint32_t b = x ? (acc[8 * h + 2 * t + 1][cc] >> 16) : (acc[8 * h + 2 * t + 1][cc] & 0xffffu);
                        w4[t] = a | (b << 16);
                    }
                    const int q = warp * (RW / 8) + h;
                    *reinterpret_cast<uint4*>(Tt + j * TT + ((q ^ key) * 8)) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
                }
            }
        __syncthreads();
        for (int idx = tid; idx < TT * (TT / 8); idx += kThreads) {
            const int j = idx / (TT / 8), c8 = idx % (TT / 8);
            const int key = (j / (2 * CP)) & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(Tt + j * TT + ((c8 ^ key) * 8));
            reinterpret_cast<uint4*>(D + (size_t)(jb + j) * NP + i0)[c8] = v;
        }
    }
    if (tid == 0 && s_dec) mark_dec(L, l, rec.task, rec.node);
}

// Upper-triangle tile pair t of an nt x nt tile grid: I <= J.
__device__ __forceinline__ void tri_pair(int t, int nt, int& I, int& J) {
    int i = 0;
    while (t >= nt - i) {
        t -= nt - i;
        ++i;
    }
    I = i;
    J = i + t;
}

// Bounded wait (thread 0 polls, the CTA follows) for slot s's compaction
// record; false after a timeout (status 1) or when another CTA recorded one.
__device__ bool wait_rec_ready(const OpenLaunch& L, int l, int s) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        const unsigned* f = reinterpret_cast<const unsigned*>(&L.rec[l][s].ready);
        int ok = 1;
        unsigned it = 0;
        while (ld_acquire(f) == 0u) {
            if (*(volatile int*)L.status != 0) { ok = 0; break; }
            if (++it > kBarrierPolls) { atomicCAS(L.status, 0, 1); ok = 0; break; }
            __nanosleep(32);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Compaction and round 0's panels of level l as one phase: the compaction
// units (one per slot) take the first places, the panel units of round 0
// (slot x 64-column tile) the later ones and wait only for their slot's
// record - a unit of a lower place, already running, so every wait ends.
__device__ void compact_panel_phase(const OpenLaunch& L, int l, int N, int* s_unit, unsigned char* smem) {
    const int tiles = L.geo[l].NP / 64;
    const int units = N + N * tiles;
    for (int u = next_unit(L, s_unit); u < units; u = next_unit(L, s_unit)) {
        if (u < N) {
            compact_unit(L, l, u);
            continue;
        }
        const int v = u - N, s = v / tiles;
        if (!wait_rec_ready(L, l, s)) return;  // the next barrier ends the launch
        panel_unit(L, l, s, (v % tiles) * 64, 0, smem);
    }
}

// Stage t of level l's closure (t = 1 .. rounds; stage 0 is compact_panel_phase) as one phase: the panel
// units of round t (slot x 64-column tile; none in the last stage) take the
// lower tickets, the update units of round t - 1 (slot x upper-triangle tile
// pair; none in stage 0) the higher ones.  The panel of round t applies
// round t - 1's update to its own pivot rows, so the two run side by side;
// the grid barrier after the stage orders round t - 1's update before round
// t's (both write the same tiles) and publishes round t's panel.
__device__ void stage_phase(const OpenLaunch& L, int l, int N, int t, int rounds, int* s_unit,
                            unsigned char* smem) {
    const int NP = L.geo[l].NP;
    const int NT = 64;  // panel tiles of 64 columns: many short units
    const int tiles = NP / NT;
    const int TT = NP >= 128 ? 128 : 64;
    const int nt = NP / TT;
    const int per = nt * (nt + 1) / 2;
    const int n_panel = t < rounds ? N * tiles : 0;
    const int units = n_panel + (t > 0 ? N * per : 0);
    for (int u = next_unit(L, s_unit); u < units; u = next_unit(L, s_unit)) {
        if (u < n_panel) {
            panel_unit(L, l, u / tiles, (u % tiles) * NT, t, smem);
            continue;
        }
        const int v = u - n_panel;
        const int s = v / per;
        int I, J;
        tri_pair(v % per, nt, I, J);
        if (TT == 128) update_unit<16, 2>(L, l, s, I, J, t - 1, smem);
        else update_unit<8, 1>(L, l, s, I, J, t - 1, smem);
    }
}

// ---------------------------------------------------------------------------
// Levels whose matrices fit in shared memory (NP <= 128: leaves of b <= 11,
// the lowest node levels): one unit per slot does the whole update of its
// matrix in shared memory - the child-summary decreases, the edge / seam
// list, the pivot compaction and every closure round (pivot block,
// panel, full update) - and writes the matrix back once.  One phase per
// level instead of 2 + 2 x rounds.
// ---------------------------------------------------------------------------
template <int RW, int CP>
__device__ void small_unit(const OpenLaunch& L, int l, int s, unsigned char* smem) {
    constexpr int NP = 8 * RW;
    static_assert(NP == 64 * CP, "square matrix of 8 warps x RW rows and 32 lanes x CP pairs");
    const OpenLevelGeom& G = L.geo[l];
    const int4 e = ld_slot(L.slots[l] + s);
    const OpenTask& T = L.tasks[e.x];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint16_t* Dg = node_mat(T.lv[l], e.y, NP);
    uint16_t* Dm = reinterpret_cast<uint16_t*>(smem);                               // [NP][NP]
    uint16_t* Pm = Dm + NP * NP;                                                     // [B][NP]
    uint16_t (*Ts)[kTLD] = reinterpret_cast<uint16_t (*)[kTLD]>(Pm + B * NP);       // [B][kTLD]
    int* kl = reinterpret_cast<int*>(&Ts[B][0]);                                     // [NP]
    uint8_t* fl = reinterpret_cast<uint8_t*>(kl + NP);                               // [NP]
    uint8_t* cls = fl + NP;                                                          // [B][kWarps]
    __shared__ int s_dec, s_chg, s_np, s_k;
    __shared__ int wtot[kWarps];
    for (int idx = tid; idx < NP * NP / 8; idx += kThreads) cp_async16(Dm + idx * 8, Dg + idx * 8);
    for (int j = tid; j < NP / 4; j += kThreads) reinterpret_cast<unsigned*>(fl)[j] = 0u;
    if (tid == 0) { s_dec = 0; s_chg = 0; s_np = 0; }
    cp_async_wait_all();
    __syncthreads();
    bool dec = false, chg = false;
    if (l >= 1) {  // child-summary decreases (internal_node.cpp:343-353), as in insert_phase
        const int nx = T.lv[l].nodes_x, g = L.g, nP = G.nP, cNP = G.childNP;
        for (int q = 0; q < g * g; ++q) {
            const int child = ((e.y / nx) * g + q / g) * T.lv[l - 1].nodes_x + ((e.y % nx) * g + q % g);
            if (__ldcg(T.lv[l - 1].dstamp + child) != T.stamp) continue;  // uniform
            const uint16_t* cm = node_mat(T.lv[l - 1], child, cNP);
            constexpr int U = 4;  // a thread's loads of U entries first, then their updates
            for (int b0 = tid; b0 < nP * nP; b0 += U * kThreads) {
                uint16_t w[U];
                int ab[U];
#pragma unroll
                for (int x = 0; x < U; ++x) {
                    const int idx = b0 + x * kThreads;
                    ab[x] = -1;
                    if (idx < nP * nP) {
                        const int p = idx / nP, pp = idx - p * nP;
                        w[x] = __ldcg(cm + (size_t)G.child_ext[p] * cNP + G.child_ext[pp]);
                        ab[x] = (q * nP + p) * NP + q * nP + pp;
                    }
                }
#pragma unroll
                for (int x = 0; x < U; ++x) {
                    if (ab[x] >= 0 && w[x] < Dm[ab[x]]) {
                        const int a = ab[x] / NP, b = ab[x] % NP;
                        Dm[ab[x]] = w[x];  // (b, a) is written by its own thread
                        fl[a] = 1;
                        fl[b] = 1;
                        dec |= G.isext[a] && G.isext[b];
                        chg = true;
                    }
                }
            }
        }
        __syncthreads();
    }
    if (warp == 0 && e.w > e.z) {  // the edge / seam list, lanes in parallel (see insert_list)
        int np = 0;
        for (int t = e.z + lane; t < e.w; t += 32) {
            const int u = L.triples[3 * t], v = L.triples[3 * t + 1];
            const uint16_t w = (uint16_t)L.triples[3 * t + 2];
            if (w < Dm[u * NP + v]) {
                Dm[u * NP + v] = w;
                Dm[v * NP + u] = w;
                const int ends[2] = {u, v};
#pragma unroll
                for (int x = 0; x < 2; ++x) {
                    const int a = ends[x];
                    const unsigned sh = (unsigned)(a & 3) * 8u;
                    const unsigned old = atomicOr(reinterpret_cast<unsigned*>(fl + (a & ~3)), 1u << sh);
                    np += ((old >> sh) & 0xffu) == 0;
                }
                dec |= G.isext[u] && G.isext[v];
                chg = true;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) np += __shfl_xor_sync(FULL, np, o);
        if (lane == 0) s_np = np;
    }
    __syncthreads();
    {   // pivot flags -> ascending list (NP <= 128 <= kThreads: one step)
        const bool on = tid < NP && fl[tid];
        const unsigned bal = __ballot_sync(FULL, on);
        if (lane == 0) wtot[warp] = __popc(bal);
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < kWarps; ++w) {
            if (w < warp) off += wtot[w];
            tot += wtot[w];
        }
        if (on) kl[off + __popc(bal & ((1u << lane) - 1u))] = tid;
        if (tid == 0) s_k = tot;
        __syncthreads();
    }
    const int k = s_k;
    if (tid == 0) {
        atomicAdd(&T.out->level[l][0], 1);
        atomicAdd(&T.out->level[l][1], k);
        atomicMax(&T.out->level[l][2], k);
        if (l == 0 && s_np) atomicAdd(&T.out->new_pivots, s_np);
        if (k) {
            const unsigned long long n = (unsigned long long)G.n;
            atomicAdd(&T.out->ops, n * n * (unsigned long long)k);
            atomicAdd(&T.out->bytes, 4ull * n * n + 4ull * (unsigned long long)k * n);
        }
    }
    for (int r = 0; r * B < k; ++r) {
        const int mk = min(B, k - r * B);
        const int* kc = kl + r * B;
        for (int idx = tid; idx < B * B; idx += kThreads) {
            const int a = idx / B, c = idx % B;
            Ts[a][c] = (a < mk && c < mk) ? Dm[kc[a] * NP + kc[c]] : (a == c ? 0 : INF);
        }
        for (int idx = tid; idx < mk * (NP / 8); idx += kThreads) {  // the pivot rows
            const int a = idx / (NP / 8), c8 = idx % (NP / 8);
            reinterpret_cast<uint4*>(Pm + a * NP)[c8] = reinterpret_cast<const uint4*>(Dm + kc[a] * NP)[c8];
        }
        __syncthreads();
        close_pivot_block(Ts, mk);
        panel_classes(Ts, mk, cls);
        __syncthreads();
        {   // the panel P = T* (x) D[Kc, :], into Pm
            uint32_t pacc[8][CP];
            panel_gemm<CP>(Ts, Pm, NP, mk, cls, pacc);
            __syncthreads();
#pragma unroll
            for (int rr = 0; rr < 8; ++rr) {
                const int a = warp * 8 + rr;
                if (a < mk)
#pragma unroll
                    for (int cc = 0; cc < CP; ++cc)
                        reinterpret_cast<uint32_t*>(Pm + a * NP + lane * 2 * CP)[cc] = pacc[rr][cc];
            }
        }
        __syncthreads();
        for (int idx = tid; idx < mk * kWarps; idx += kThreads) {  // update classes per warp row group
            const int a = idx / kWarps, w = idx % kWarps;
            uint32_t mn = 0xffffu, mx = 0;
#pragma unroll
            for (int rr = 0; rr < RW; ++rr) {
                const uint32_t v = Pm[a * NP + w * RW + rr];
                mn = min(mn, v);
                mx = max(mx, v);
            }
            cls[idx] = mn >= INF ? 0 : (mx <= INF_HEADROOM ? 1 : 2);
        }
        __syncthreads();
        // D = min(D, P^T (x) P): warp w rows RW*w.., lane CP pairs
        uint32_t acc[RW][CP];
#pragma unroll
        for (int rr = 0; rr < RW; ++rr)
#pragma unroll
            for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = INF2;
        for (int kk = 0; kk < mk; ++kk) {
            const int c = cls[kk * kWarps + warp];
            if (c == 0) continue;  // uniform over the warp
            uint32_t bv[CP];
#pragma unroll
            for (int cc = 0; cc < CP; ++cc) bv[cc] = reinterpret_cast<const uint32_t*>(Pm + kk * NP + lane * 2 * CP)[cc];
            uint32_t av[RW];
#pragma unroll
            for (int q2 = 0; q2 < RW / 2; ++q2) {
                const uint32_t w2 = reinterpret_cast<const uint32_t*>(Pm + kk * NP + warp * RW)[q2];
                av[2 * q2] = splat(w2);
                av[2 * q2 + 1] = splat(w2 >> 16);
            }
            if (c == 1) {
#pragma unroll
                for (int rr = 0; rr < RW; ++rr)
#pragma unroll
                    for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = acc_fast(acc[rr][cc], bv[cc], av[rr]);
            } else {
#pragma unroll
                for (int rr = 0; rr < RW; ++rr) {
                    const uint32_t tt = INF2 - av[rr];
#pragma unroll
                    for (int cc = 0; cc < CP; ++cc) acc[rr][cc] = acc_clamp(acc[rr][cc], bv[cc], av[rr], tt);
                }
            }
        }
        const int col = lane * 2 * CP;
        uint32_t cext[CP];
#pragma unroll
        for (int cc = 0; cc < CP; ++cc)
            cext[cc] = (G.isext[col + 2 * cc] ? 0xffffu : 0u) | (G.isext[col + 2 * cc + 1] ? 0xffff0000u : 0u);
#pragma unroll
        for (int rr = 0; rr < RW; ++rr) {
            const int row = warp * RW + rr;
            uint32_t* dp = reinterpret_cast<uint32_t*>(Dm + row * NP + col);
            const bool rext = G.isext[row] != 0;
#pragma unroll
            for (int cc = 0; cc < CP; ++cc) {
                const uint32_t o = dp[cc], nv = min2(acc[rr][cc], o);
                const uint32_t diff = nv ^ o;
                if (diff) {
                    dp[cc] = nv;
                    chg = true;
                    if (rext) dec |= (diff & cext[cc]) != 0;
                }
            }
        }
        __syncthreads();
    }
    if (__any_sync(FULL, chg) && lane == 0) s_chg = 1;
    if (__any_sync(FULL, dec) && lane == 0) s_dec = 1;
    __syncthreads();
    if (s_chg)
        for (int idx = tid; idx < NP * NP / 8; idx += kThreads)
            reinterpret_cast<uint4*>(Dg)[idx] = reinterpret_cast<const uint4*>(Dm)[idx];
    if (tid == 0) {
        T.lv[l].kcnt[e.y] = k;
        if (s_dec) mark_dec(L, l, e.x, e.y);
    }
}

__device__ void small_phase(const OpenLaunch& L, int l, int N, int* s_unit, unsigned char* smem) {
    const int NP = L.geo[l].NP;
    for (int s = next_unit(L, s_unit); s < N; s = next_unit(L, s_unit)) {
        if (NP == 128) small_unit<16, 2>(L, l, s, smem);
        else small_unit<8, 1>(L, l, s, smem);
    }
}

constexpr size_t kPanelSmem = (size_t)3 * B * kTLD * sizeof(uint16_t) + (size_t)B * 64 * sizeof(uint16_t) +
                              B * sizeof(int) + (size_t)B * kWarps;
constexpr size_t kUpdateSmem = (size_t)B * 128 * (sizeof(uint32_t) + sizeof(uint16_t)) + (size_t)B * kWarps +
                               (size_t)128 * 128 * sizeof(uint16_t);
constexpr size_t kTransposeSmem = (size_t)128 * (128 + 8) * sizeof(uint16_t);
constexpr size_t kOpenSmem = std::max(std::max(kPanelSmem, (size_t)kInsertSmem), std::max(kUpdateSmem, kTransposeSmem));

// SM-aware order of the CTAs, for the units a CTA takes without a ticket:
// the first CTA to start on each SM gets places 0 .. S - 1 (S SMs), the
// others the places after them, so a phase of at most S units runs one unit
// per SM (the block scheduler puts blocks b and b + 6 on one SM, for
// instance).  sm_arrive runs at launch, sm_order after the first barrier.
__device__ __forceinline__ void sm_arrive(const OpenLaunch& L, int* s_unit) {
    if (threadIdx.x != 0) return;
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    int first = 0;
    if (smid < (unsigned)kOpenSmSlots) first = atomicAdd(L.sm + 3 + smid, 1u) == 0;
    else atomicOr(L.sm + 2, 1u);
    s_unit[3] = (int)blockIdx.x;
    s_unit[4] = first;
    s_unit[5] = (int)atomicAdd(L.sm + (first ? 0 : 1), 1u);
}
__device__ __forceinline__ void sm_order(const OpenLaunch& L, int* s_unit) {
    if (threadIdx.x != 0) return;
    if (__ldcg(L.sm + 2) != 0u) return;  // an SM id beyond the table: launch order
    s_unit[3] = s_unit[4] ? s_unit[5] : (int)__ldcg(L.sm) + s_unit[5];
}

__global__ void __launch_bounds__(kThreads, 2) open_persistent_kernel(const OpenLaunch L) {
    extern __shared__ __align__(16) unsigned char osm[];
    __shared__ int s_unit[6];
    if (threadIdx.x == 0) {
        s_unit[1] = -1;
        s_unit[2] = 0;
    }
    int phase = 0;
    const bool stamp = L.trace && blockIdx.x == 0 && threadIdx.x == 0;
    if (stamp) L.trace[0] = global_timer();
    auto end_phase = [&]() -> bool {
        const bool ok = open_barrier(L, phase, s_unit);
        if (stamp && phase < kOpenTrace - 1) L.trace[1 + phase] = global_timer();
        ++phase;
        return ok;
    };
    sm_arrive(L, s_unit);
    stamp_phase(L);
    if (!end_phase()) return;
    sm_order(L, s_unit);  // visible to the CTA at next_unit's barrier
    for (int l = 0; l <= L.maxH; ++l) {
        const int N = min(*(volatile int*)(L.count + l), L.cap[l]);
        if (N == 0) continue;
        if (L.geo[l].NP <= 128) {  // the whole level in one phase, one matrix per unit
            small_phase(L, l, N, s_unit, osm);
            if (!end_phase()) return;
            continue;
        }
        insert_phase(L, l, N, s_unit, osm);
        if (!end_phase()) return;
        compact_panel_phase(L, l, N, s_unit, osm);  // stage 0 of the closure with the compaction
        if (!end_phase()) return;
        const int rounds = (*(volatile int*)(L.maxk + l) + B - 1) / B;
        for (int t = 1; rounds > 0 && t <= rounds; ++t) {
            stage_phase(L, l, N, t, rounds, s_unit, osm);
            if (!end_phase()) return;
        }
    }
}

}  // namespace

// Dirty levels of an incremental query: viewpoint j (sorted order, leaf
// vp0[4 j]) gets 1 + the lowest level whose matrix on its leaf-to-root chain
// was listed by an opening call after the stamp `seen` (stamps compare modulo
// 2^32), 0 when none was: its projections below that level are unchanged.
__global__ void incremental_dirty_kernel(const int* __restrict__ vp0, int ns, IncrementalChain C, unsigned seen,
                                         uint8_t* dirty, int* n_dirty) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    const int leaf = vp0[4 * j];
    int tx = leaf % C.leaves_x, ty = leaf / C.leaves_x;
    int lo = -1;
    for (int l = 0; l <= C.H && lo < 0; ++l) {
        if (l > 0) {
            tx /= C.g;
            ty /= C.g;
        }
        if ((int)(C.mstamp[l][ty * C.nodes_x[l] + tx] - seen) > 0) lo = l;
    }
    dirty[j] = (uint8_t)(lo + 1);
    if (lo >= 0) atomicAdd(n_dirty, 1);
}

void launch_incremental_dirty(const int* vp0, int ns, const IncrementalChain& C, unsigned seen, uint8_t* dirty,
                              int* n_dirty, cudaStream_t st) {
    if (ns <= 0) return;
    incremental_dirty_kernel<<<(ns + 255) / 256, 256, 0, st>>>(vp0, ns, C, seen, dirty, n_dirty);
}

size_t open_smem_bytes() { return kOpenSmem; }

int open_grid_blocks(int device) {
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(open_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kOpenSmem);
        configured = true;
    }
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, open_persistent_kernel, kThreads, kOpenSmem);
    return sms * std::max(1, std::min(per, 2));
}

cudaError_t launch_open(const OpenLaunch& L, int grid, cudaStream_t st) {
    void* args[] = {const_cast<OpenLaunch*>(&L)};
    return cudaLaunchCooperativeKernel((const void*)open_persistent_kernel, dim3(grid), dim3(kThreads), args,
                                       kOpenSmem, st);
}

}  // namespace hb
