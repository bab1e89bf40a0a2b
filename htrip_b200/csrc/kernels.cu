// sm_100a kernels of the HTRIP min-plus hierarchy.
//
// Layout: every tropical matrix (leaf D, node D_U) is a dense row-major u16
// square of logical order n padded to NP (multiple of 64) with INF in the
// padding; matrix m of a level lives at base + m*NP*NP.  All arithmetic is
// the exact clamped min-plus of minplus.cuh, so every result is identical to
// the reference's scalar / AVX2 arithmetic.
#include "kernels.cuh"
#include "minplus.cuh"

#include <algorithm>

namespace hb {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// grid.y / grid.z are limited to 65535: per-matrix launches go in slices.
constexpr int kMaxGridY = 65535;

__device__ __forceinline__ uint16_t* mat_ptr(const MatSet& M, int m) {
    return M.base + (size_t)m * M.NP * M.NP;
}

// ---------------------------------------------------------------------------
// Leaf APSP: one warp per source cell, bit-parallel BFS.  Lane r owns row r
// of the b x b leaf as a bitmask; a BFS level is one shift/shuffle step, so
// the BFS level number is the reference's BFS distance (leaf_tile.cpp:111-152).
// Non-passable sources keep the tropical identity row (leaf_tile.cpp:66-68).
// ---------------------------------------------------------------------------
constexpr int kBfsWarps = 8;

__global__ void __launch_bounds__(kBfsWarps * 32)
leaf_bfs_kernel(const uint8_t* __restrict__ pass, int S, int b, int leaves_x, MatSet L, const int* __restrict__ list,
                int y0) {
    extern __shared__ __align__(16) uint16_t sm_rows[];
    const int leaf = list ? list[y0 + blockIdx.y] : y0 + blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int src = blockIdx.x * kBfsWarps + warp;
    const int NP = L.NP, n = b * b;
    if (src >= NP) return;
    uint16_t* row = sm_rows + (size_t)warp * NP;
    const int ty = leaf / leaves_x, tx = leaf % leaves_x;
    const int R0 = ty * b, C0 = tx * b;
    uint32_t m = 0;
    if (lane < b) {
        const uint8_t* p = pass + (size_t)(R0 + lane) * S + C0;
        for (int c = 0; c < b; ++c) m |= (uint32_t)(p[c] != 0) << c;
    }
    for (int j = lane; j < NP; j += 32) row[j] = INF;
    __syncwarp();
    if (src < n) {
        const int sr = src / b, sc = src % b;
        const uint32_t srow = __shfl_sync(FULL, m, sr);
        if (lane == 0) row[src] = 0;
        if ((srow >> sc) & 1u) {
            const uint32_t rowmask = (b == 32) ? FULL : ((1u << b) - 1u);
            uint32_t vis = (lane == sr) ? (1u << sc) : 0u;
            uint32_t front = vis;
            for (int d = 1;; ++d) {
                uint32_t up = __shfl_up_sync(FULL, front, 1);
                uint32_t dn = __shfl_down_sync(FULL, front, 1);
                if (lane == 0) up = 0;
                if (lane == 31) dn = 0;
                const uint32_t nb = ((front << 1) | (front >> 1) | up | dn) & rowmask;
                uint32_t nw = nb & m & ~vis;
                vis |= nw;
                front = nw;
                if (!__any_sync(FULL, nw)) break;
                while (nw) {
                    const int c = __ffs(nw) - 1;
                    nw &= nw - 1;
                    row[lane * b + c] = (uint16_t)d;
                }
            }
        }
    }
    __syncwarp();
    uint4* dst = reinterpret_cast<uint4*>(mat_ptr(L, leaf) + (size_t)src * NP);
    const uint4* s4 = reinterpret_cast<const uint4*>(row);
    for (int j = lane; j < NP / 8; j += 32) dst[j] = s4[j];
}

// ---------------------------------------------------------------------------
// Node initial D_U (internal_node.cpp:98-145): entry (i, j) of node n is the
// child summary S_q[p][p'] when i = q*nP + p and j = q*nP + p' lie in the
// same child block q, INF otherwise (and in the padding).  S_q is the child
// matrix restricted to its exterior ports: child[ext[p]][ext[p']].
// ---------------------------------------------------------------------------
__global__ void node_init_kernel(MatSet N, MatSet Cm, const int* __restrict__ cext, int nP, int g,
                                 int nodes_x, int child_nodes_x, const int* __restrict__ list, int y0) {
    const int node = list ? list[y0 + blockIdx.y] : y0 + blockIdx.y;
    const int NP = N.NP, nV = N.n;
    const size_t chunk = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // 8 entries
    const size_t per_row = NP / 8;
    if (chunk >= (size_t)NP * per_row) return;
    const int i = (int)(chunk / per_row);
    const int j0 = (int)(chunk % per_row) * 8;
    uint16_t v[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) v[t] = INF;
    if (i < nV) {
        const int q = i / nP, p = i - q * nP;
        const int tx = node % nodes_x, ty = node / nodes_x;
        const int cx = q % g, cy = q / g;
        const int child = (ty * g + cy) * child_nodes_x + (tx * g + cx);
        const uint16_t* crow = mat_ptr(Cm, child) + (size_t)cext[p] * Cm.NP;
        const int lo = q * nP, hi = lo + nP;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int j = j0 + t;
            if (j >= lo && j < hi) v[t] = crow[cext[j - lo]];
        }
    }
    uint4 o;
    o.x = v[0] | ((uint32_t)v[1] << 16);
    o.y = v[2] | ((uint32_t)v[3] << 16);
    o.z = v[4] | ((uint32_t)v[5] << 16);
    o.w = v[6] | ((uint32_t)v[7] << 16);
    reinterpret_cast<uint4*>(mat_ptr(N, node) + (size_t)i * NP)[j0 / 8] = o;
}

// Build-time seams: both cells Free -> unit edge, both endpoints are pivots.
__global__ void seams_build_kernel(MatSet N, const int* __restrict__ seams, int n_seams,
                                   const uint8_t* __restrict__ pass, const uint16_t* __restrict__ wts, int S,
                                   int side, int nodes_x, uint8_t* kflag, const int* __restrict__ list, int y0) {
    const int node = list ? list[y0 + blockIdx.y] : y0 + blockIdx.y;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_seams) return;
    const int* e = seams + 6 * s;
    const int R0 = (node / nodes_x) * side, C0 = (node % nodes_x) * side;
    const size_t a = (size_t)(R0 + e[2]) * S + C0 + e[3], c = (size_t)(R0 + e[4]) * S + C0 + e[5];
    if (!pass[a] || !pass[c]) return;
    const uint16_t w = wts ? edge_weight(wts[a], wts[c]) : (uint16_t)1;  // internal_node.cpp:160-161
    if (w >= INF) return;
    uint16_t* D = mat_ptr(N, node);
    const int NP = N.NP;
    D[(size_t)e[0] * NP + e[1]] = min(D[(size_t)e[0] * NP + e[1]], w);
    D[(size_t)e[1] * NP + e[0]] = min(D[(size_t)e[1] * NP + e[0]], w);
    kflag[(size_t)node * NP + e[0]] = 1;
    kflag[(size_t)node * NP + e[1]] = 1;
}

// ---------------------------------------------------------------------------
// Weighted leaf (LeafTile::recomputeFromGrid's Dijkstra branch,
// leaf_tile.cpp:154-192): D starts as the tile's weighted adjacency - 0 on
// the diagonal, w(u, v) between 4-adjacent passable cells, INF elsewhere and
// in the padding - and every passable cell becomes a pivot; the closure over
// those pivots is the all-pairs shortest-path matrix, equal to the
// saturated Dijkstra result.  One warp per matrix row.
// ---------------------------------------------------------------------------
__global__ void leaf_weight_init_kernel(const uint8_t* __restrict__ pass, const uint16_t* __restrict__ wts, int S,
                                        int b, int leaves_x, MatSet L, uint8_t* kflag, const int* __restrict__ list,
                                        int y0) {
    const int leaf = list ? list[y0 + blockIdx.y] : y0 + blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int src = blockIdx.x * (blockDim.x >> 5) + warp;
    const int NP = L.NP, n = b * b;
    if (src >= NP) return;
    uint16_t* row = mat_ptr(L, leaf) + (size_t)src * NP;
    const uint4 inf4 = make_uint4(INF2, INF2, INF2, INF2);
    for (int j = lane; j < NP / 8; j += 32) reinterpret_cast<uint4*>(row)[j] = inf4;
    __syncwarp();
    if (lane != 0) return;
    uint8_t* f = kflag + (size_t)leaf * NP + src;
    if (src >= n) {
        *f = 0;
        return;
    }
    row[src] = 0;
    const int R0 = (leaf / leaves_x) * b, C0 = (leaf % leaves_x) * b;
    const int sr = src / b, sc = src % b;
    const size_t cu = (size_t)(R0 + sr) * S + C0 + sc;
    const bool pu = pass[cu] != 0;
    *f = pu ? 1 : 0;
    if (!pu) return;
    const int dr[4] = {-1, 1, 0, 0}, dc[4] = {0, 0, -1, 1};
    for (int d = 0; d < 4; ++d) {
        const int vr = sr + dr[d], vc = sc + dc[d];
        if (vr < 0 || vr >= b || vc < 0 || vc >= b) continue;
        const size_t cv = (size_t)(R0 + vr) * S + C0 + vc;
        if (!pass[cv]) continue;
        const uint16_t w = edge_weight(wts[cu], wts[cv]);
        if (w < INF) row[vr * b + vc] = w;
    }
}

// ---------------------------------------------------------------------------
// Pivot compaction: flags -> ascending index list, one CTA per matrix.
// ---------------------------------------------------------------------------
__global__ void compact_pivots_kernel(const Slot* __restrict__ S, int NP, int* slot_cnt) {
    __shared__ int warp_tot[32];
    __shared__ int base;
    const Slot& sl = S[blockIdx.x];
    uint8_t* f = sl.kflag;
    int* out = sl.klist;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (int j0 = 0; j0 < NP; j0 += blockDim.x) {
        const int j = j0 + threadIdx.x;
        const bool on = j < NP && f[j];
        const unsigned bal = __ballot_sync(FULL, on);
        if (lane == 0) warp_tot[warp] = __popc(bal);
        __syncthreads();
        int off = base;
        for (int w = 0; w < warp; ++w) off += warp_tot[w];
        if (on) {
            out[off + __popc(bal & ((1u << lane) - 1u))] = j;
            f[j] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < nw; ++w) t += warp_tot[w];
            base += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *sl.kcnt = base;
        if (slot_cnt) slot_cnt[blockIdx.x] = base;
    }
}

// ---------------------------------------------------------------------------
// Blocked pivot-set Kleene closure, one round over pivots Kc (|Kc| = mk <= B):
//   T  = D[Kc, Kc], closed once per matrix in shared memory
//        (pivot_close_kernel, Floyd-Warshall over Kc),
//   R' = T* (x) D[Kc, :]                (closure_gemm_kernel<.., true>,
//                                        B x NP per matrix)
//   D  = min(D, R'^T (x) R')            (closure_gemm_kernel<.., false>; D
//                                        is symmetric, so
//                                        R'[k][i] = (D[:,Kc] (x) T*)[i][k])
// This is exactly the reference's sequential relaxation over the same pivots
// (leaf_tile.cpp:348-371, internal_node.cpp:201-231, :372-399): both give
// the unique shortest-path closure through the pivot set.
// ---------------------------------------------------------------------------
// Closure of the round's pivot block T = D[Kc, Kc] (mk <= B) of every
// active matrix, once per matrix: Floyd-Warshall over Kc in shared memory
// (the reference's sequential relaxation restricted to the pivots).  tstar
// receives T* as a B x B block (identity beyond mk); T is symmetric, so T*
// is too.
__global__ void __launch_bounds__(256)
pivot_close_kernel(const Slot* __restrict__ S, int NP, int round, uint16_t* tstar) {
    constexpr int B = kPivotChunk;   // 64: 256 threads x 16 entries
    constexpr int LD = B + 8;        // padded row (144 bytes): column reads hit distinct banks
    __shared__ __align__(16) uint16_t T[B][LD];
    __shared__ int kc[B];
    const int slot = blockIdx.x;
    const Slot& sl = S[slot];
    const int mk = min(B, *sl.kcnt - round * B);
    if (mk <= 0) return;
    const int* K = sl.klist + round * B;
    const uint16_t* D = sl.mat;
    const int tid = threadIdx.x;
    if (tid < mk) kc[tid] = K[tid];
    __syncthreads();
    for (int idx = tid; idx < B * B; idx += blockDim.x) {
        const int a = idx / B, c = idx % B;
        T[a][c] = (a < mk && c < mk) ? D[(size_t)kc[a] * NP + kc[c]] : (a == c ? 0 : INF);
    }
    __syncthreads();
    // Thread t owns row a = t / 4, columns c0 .. c0 + 15 (8 packed pairs).
    const int a = tid >> 2, c0 = (tid & 3) * 16;
    uint32_t v[8];
    {
        const uint4 x = *reinterpret_cast<const uint4*>(&T[a][c0]);
        const uint4 y = *reinterpret_cast<const uint4*>(&T[a][c0 + 8]);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w; v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
    }
    // Step kk reads only row kk and column kk, which step kk leaves unchanged
    // (T[kk][kk] = 0), so one barrier per step orders the writes of step kk
    // before the reads of step kk + 1.
    for (int kk = 0; kk < mk; ++kk) {
        const uint32_t t = T[a][kk];
        const uint4 x = *reinterpret_cast<const uint4*>(&T[kk][c0]);
        const uint4 y = *reinterpret_cast<const uint4*>(&T[kk][c0 + 8]);
        if (t < INF) {
            const uint32_t r[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
            const uint32_t aa = splat(t), tt = splat(INF - t);
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = acc_clamp(v[i], r[i], aa, tt);
            *reinterpret_cast<uint4*>(&T[a][c0]) = make_uint4(v[0], v[1], v[2], v[3]);
            *reinterpret_cast<uint4*>(&T[a][c0 + 8]) = make_uint4(v[4], v[5], v[6], v[7]);
        }
        __syncthreads();
    }
    uint4* out = reinterpret_cast<uint4*>(tstar + (size_t)slot * B * B + (size_t)a * B + c0);
    out[0] = make_uint4(v[0], v[1], v[2], v[3]);
    out[1] = make_uint4(v[4], v[5], v[6], v[7]);
}

// Register-tiled symmetric rank-|Kc| min-plus update.  Warp w owns RW rows
// of the CTA tile; all 32 lanes of a warp share those rows, so the pivot
// value a = R'[k][row] is warp-uniform and the fast / clamped / skip choice
// never diverges.  Each lane owns CP packed column pairs.
//
// PANEL = true computes the round's panel with the same tiling instead:
//   R'[a][j] = min_c T*[c][a] (+) D[Kc[c]][j]      (T* symmetric, so
// T*[c][a] = T*[a][c]), one CTA per 64*CP columns and all B pivot rows,
// and marks the 64-column tiles of R' holding any finite value.
template <int RW, int CP, bool PANEL>
__global__ void __launch_bounds__(256)
closure_gemm_kernel(const Slot* __restrict__ S, int NP, int round, uint16_t* panel, uint8_t* flags,
                    const uint16_t* __restrict__ tstar) {
    constexpr int B = kPivotChunk;
    constexpr int MT = 8 * RW;
    constexpr int NT = 64 * CP;
    static_assert(!PANEL || MT == B, "the panel tile covers all pivot rows");
    extern __shared__ __align__(16) uint16_t sm[];
    uint16_t* As = sm;            // [B][MT]
    uint16_t* Bs = sm + B * MT;   // [B][NT]
    __shared__ int kc[B];
    __shared__ int tile_any[NT / kFlagTile];
    const int slot = blockIdx.z;
    const Slot& sl = S[slot];
    const int mk = min(B, *sl.kcnt - round * B);
    if (mk <= 0) return;
    const int i0 = blockIdx.y * MT, j0 = blockIdx.x * NT;
    uint16_t* P = panel + (size_t)slot * B * NP;
    uint16_t* D = sl.mat;
    const int tid = threadIdx.x;
    if constexpr (PANEL) {
        const int* K = sl.klist + round * B;
        if (tid < mk) kc[tid] = K[tid];
        if (tid < NT / kFlagTile) tile_any[tid] = 0;
        __syncthreads();
        const uint16_t* Ts = tstar + (size_t)slot * B * B;
        for (int idx = tid; idx < mk * (MT / 8); idx += blockDim.x) {
            const int a = idx / (MT / 8), c8 = idx % (MT / 8);
            reinterpret_cast<uint4*>(As + a * MT)[c8] = reinterpret_cast<const uint4*>(Ts + (size_t)a * B)[c8];
        }
        for (int idx = tid; idx < mk * (NT / 8); idx += blockDim.x) {
            const int a = idx / (NT / 8), c8 = idx % (NT / 8);
            reinterpret_cast<uint4*>(Bs + a * NT)[c8] =
                reinterpret_cast<const uint4*>(D + (size_t)kc[a] * NP + j0)[c8];
        }
    } else {
        const uint8_t* fl = flags + (size_t)slot * (NP / kFlagTile);
        bool any_i = false, any_j = false;
        for (int t = 0; t < MT / kFlagTile + (MT % kFlagTile ? 1 : 0); ++t) any_i |= fl[(i0 + t * kFlagTile) / kFlagTile] != 0;
        for (int t = 0; t < NT / kFlagTile + (NT % kFlagTile ? 1 : 0); ++t) any_j |= fl[(j0 + t * kFlagTile) / kFlagTile] != 0;
        if (!any_i || !any_j) return;
        for (int idx = tid; idx < mk * (MT / 8); idx += blockDim.x) {
            const int a = idx / (MT / 8), c8 = idx % (MT / 8);
            reinterpret_cast<uint4*>(As + a * MT)[c8] = reinterpret_cast<const uint4*>(P + (size_t)a * NP + i0)[c8];
        }
        for (int idx = tid; idx < mk * (NT / 8); idx += blockDim.x) {
            const int a = idx / (NT / 8), c8 = idx % (NT / 8);
            reinterpret_cast<uint4*>(Bs + a * NT)[c8] = reinterpret_cast<const uint4*>(P + (size_t)a * NP + j0)[c8];
        }
    }
    const int warp = tid >> 5, lane = tid & 31;
    uint32_t acc[RW][CP];
    const int col = j0 + lane * 2 * CP;
#pragma unroll
    for (int r = 0; r < RW; ++r) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(D + (size_t)(i0 + warp * RW + r) * NP + col);
#pragma unroll
        for (int c = 0; c < CP; ++c) acc[r][c] = PANEL ? INF2 : src[c];
    }
    __syncthreads();
    for (int k = 0; k < mk; ++k) {
        uint32_t bv[CP];
#pragma unroll
        for (int c = 0; c < CP; ++c) bv[c] = reinterpret_cast<const uint32_t*>(Bs + k * NT + lane * 2 * CP)[c];
        const uint16_t* arow = As + k * MT + warp * RW;
#pragma unroll
        for (int r = 0; r < RW; ++r) {
            const uint32_t a = arow[r];
            if (a <= INF_HEADROOM) {
                const uint32_t aa = splat(a);
#pragma unroll
                for (int c = 0; c < CP; ++c) acc[r][c] = acc_fast(acc[r][c], bv[c], aa);
            } else if (a < INF) {
                const uint32_t aa = splat(a), tt = splat(INF - a);
#pragma unroll
                for (int c = 0; c < CP; ++c) acc[r][c] = acc_clamp(acc[r][c], bv[c], aa, tt);
            }
        }
    }
    if constexpr (PANEL) {
        bool any = false;
#pragma unroll
        for (int r = 0; r < RW; ++r) {
            uint32_t* dst = reinterpret_cast<uint32_t*>(P + (size_t)(warp * RW + r) * NP + col);
#pragma unroll
            for (int c = 0; c < CP; ++c) {
                dst[c] = acc[r][c];
                any |= acc[r][c] != INF2;
            }
        }
        if (any) tile_any[(lane * 2 * CP) / kFlagTile] = 1;
        __syncthreads();
        if (tid < NT / kFlagTile) flags[(size_t)slot * (NP / kFlagTile) + j0 / kFlagTile + tid] = tile_any[tid] ? 1 : 0;
    } else {
#pragma unroll
        for (int r = 0; r < RW; ++r) {
            uint32_t* dst = reinterpret_cast<uint32_t*>(D + (size_t)(i0 + warp * RW + r) * NP + col);
#pragma unroll
            for (int c = 0; c < CP; ++c) dst[c] = acc[r][c];
        }
    }
}

// ---------------------------------------------------------------------------
// Incremental inserts.
// ---------------------------------------------------------------------------
// In-leaf edges, processed sequentially per leaf like the reference loop
// (leaf_tile.cpp:311-330): an edge counts (and its endpoints become pivots)
// only if it shortens D[u][v].  Edges of slot s: list[list_begin .. list_end).
__global__ void leaf_edges_kernel(const Slot* __restrict__ S, const int* __restrict__ edges, int NP,
                                  int* task_pivots) {
    if (threadIdx.x != 0) return;
    const Slot& sl = S[blockIdx.x];
    uint16_t* D = sl.mat;
    uint8_t* f = sl.kflag;
    int np = 0;
    for (int e = sl.list_begin; e < sl.list_end; ++e) {
        const int u = edges[3 * e], v = edges[3 * e + 1];
        const uint16_t w = (uint16_t)edges[3 * e + 2];
        if (w < D[(size_t)u * NP + v]) {
            D[(size_t)u * NP + v] = w;
            D[(size_t)v * NP + u] = w;
            if (!f[u]) { f[u] = 1; ++np; }
            if (!f[v]) { f[v] = 1; ++np; }
        }
    }
    atomicAdd(task_pivots + sl.task, np);
}

// Child-summary decreases (internal_node.cpp:343-353).  Inserting every child
// summary entry that is smaller than the parent's is the same as inserting
// the reference's decrease list: entries that did not decrease can never be
// smaller than the parent's (the parent block is <= the old summary).
__global__ void node_child_insert_kernel(const Slot* __restrict__ S, const int* __restrict__ cext, int nP, int g,
                                         int NP, int childNP) {
    const Slot& sl = S[blockIdx.z];
    const int q = blockIdx.y;
    const int tx = sl.node % sl.nodes_x, ty = sl.node / sl.nodes_x;
    const int child = (ty * g + q / g) * sl.child_nodes_x + (tx * g + q % g);
    if (!sl.child_dec[child]) return;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)nP * nP) return;
    const int p = (int)(idx / nP), pp = (int)(idx % nP);
    const uint16_t w = sl.child_mat[((size_t)child * childNP + cext[p]) * childNP + cext[pp]];
    uint16_t* D = sl.mat;
    const int u = q * nP + p, v = q * nP + pp;
    if (w < D[(size_t)u * NP + v]) {
        D[(size_t)u * NP + v] = w;  // (v, u) is written by its own thread
        sl.kflag[u] = 1;
        sl.kflag[v] = 1;
    }
}

// Update-time seams (internal_node.cpp:356-365), sequential per node; seams
// of slot s: list[list_begin .. list_end).
__global__ void node_seams_kernel(const Slot* __restrict__ S, const int* __restrict__ seams, int NP) {
    if (threadIdx.x != 0) return;
    const Slot& sl = S[blockIdx.x];
    uint16_t* D = sl.mat;
    for (int s = sl.list_begin; s < sl.list_end; ++s) {
        const int u = seams[3 * s], v = seams[3 * s + 1];
        const uint16_t w = (uint16_t)seams[3 * s + 2];
        if (w < D[(size_t)u * NP + v]) {
            D[(size_t)u * NP + v] = w;
            D[(size_t)v * NP + u] = w;
            sl.kflag[u] = 1;
            sl.kflag[v] = 1;
        }
    }
}

// Exterior block snapshot of every non-root slot (summary S / S_U before the
// update).
__global__ void ext_snapshot_kernel(const Slot* __restrict__ S, const int* __restrict__ ext, int nExt, int NP,
                                    uint16_t* snap) {
    const int slot = blockIdx.y;
    if (S[slot].root) return;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)nExt * nExt) return;
    const int a = (int)(idx / nExt), c = (int)(idx % nExt);
    snap[(size_t)slot * nExt * nExt + idx] = S[slot].mat[(size_t)ext[a] * NP + ext[c]];
}

// After the update: a non-root slot whose exterior block decreased anywhere
// gets its decrease flag (and slot_dec[slot]) set (refreshBoundarySummary,
// leaf_tile.cpp:253-273, internal_node.cpp:415-433).  Every node slot also
// clears its children's decrease flags, which its insert stage has consumed:
// outside an opening call all decrease flags are zero.
__global__ void ext_compare_kernel(const Slot* __restrict__ S, const int* __restrict__ ext, int nExt, int NP,
                                   const uint16_t* __restrict__ snap, uint8_t* slot_dec, int g, int any_change) {
    const int slot = blockIdx.y;
    const Slot& sl = S[slot];
    if (any_change) {  // rebuilds: slot_dec[slot] = 1 when any exterior entry differs, nothing else
        const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        bool d = false;
        if (idx < (size_t)nExt * nExt) {
            const int a = (int)(idx / nExt), c = (int)(idx % nExt);
            d = sl.mat[(size_t)ext[a] * NP + ext[c]] != snap[(size_t)slot * nExt * nExt + idx];
        }
        if (__any_sync(FULL, d) && (threadIdx.x & 31) == 0) slot_dec[slot] = 1;
        return;
    }
    if (sl.child_dec && blockIdx.x == 0 && threadIdx.x < g * g) {
        const int q = threadIdx.x;
        const int tx = sl.node % sl.nodes_x, ty = sl.node / sl.nodes_x;
        sl.child_dec[(ty * g + q / g) * sl.child_nodes_x + (tx * g + q % g)] = 0;
    }
    if (sl.root) return;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool d = false;
    if (idx < (size_t)nExt * nExt) {
        const int a = (int)(idx / nExt), c = (int)(idx % nExt);
        d = sl.mat[(size_t)ext[a] * NP + ext[c]] < snap[(size_t)slot * nExt * nExt + idx];
    }
    if (__any_sync(FULL, d) && (threadIdx.x & 31) == 0) {
        *sl.dec = 1;
        slot_dec[slot] = 1;
    }
}

__global__ void gather_block_kernel(const uint16_t* __restrict__ mat, int NP, const int* __restrict__ rows, int nr,
                                    const int* __restrict__ cols, int nc, uint16_t* out) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)nr * nc) return;
    const int a = (int)(idx / nc), c = (int)(idx % nc);
    out[idx] = mat[(size_t)rows[a] * NP + cols[c]];
}

// Canonical checksum of a matrix family: the sum (mod 2^64) over matrices m
// and logical entries (i, j), i, j < n, of splitmix64(((m*n + i)*n + j) << 16
// | D[i][j]).  Padding is excluded, so the digest depends only on the
// matrices' contents, never on the layout.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void __launch_bounds__(256) digest_kernel(MatSet M, int count, unsigned long long* out) {
    const int n = M.n, NP = M.NP;
    const size_t rows = (size_t)count * n;
    unsigned long long acc = 0;
    for (size_t r = blockIdx.x; r < rows; r += gridDim.x) {
        const size_t m = r / n, i = r % n;
        const uint16_t* row = M.base + (m * NP + i) * NP;
        for (int j = threadIdx.x; j < n; j += blockDim.x) acc += mix64(((r * n + j) << 16) | row[j]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// Register-only rate of the packed-u16 min-plus update, 16 entries per
// thread per iteration on 8 independent accumulators.  Variants:
//   0  clamped: min2(add2(min2(b, INF - a), a), c)      (any a <= INF)
//   1  clamped with the fused add+min (__viaddmin_u16x2)
//   2  fast:    min2(add2(b, a), c)                      (a <= 5535)
//   3  fast with the fused add+min
//   4  saturating: min2(vaddus2(b, a), c) (any a <= INF: a sum above 65535
//      saturates, and min with c <= INF gives the clamped result)
// Operands stay below 16384, so no variant wraps.
template <int V>
__global__ void __launch_bounds__(512) minplus_rate_kernel(int iters, uint32_t seed, uint32_t* sink) {
    uint32_t acc[8], bv[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        acc[c] = INF2 - (threadIdx.x + c);
        bv[c] = ((seed * (c + 1) + threadIdx.x) & 0x3FFFu) * 0x10001u;
    }
    uint32_t a = (threadIdx.x * 7u + seed) & 0x3FFFu;
    for (int i = 0; i < iters; ++i) {
        const uint32_t aa = splat(a);
        const uint32_t tt = INF2 - aa;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if constexpr (V == 0) acc[c] = min2(add2(min2(bv[c], tt), aa), acc[c]);
            else if constexpr (V == 1) acc[c] = __viaddmin_u16x2(min2(bv[c], tt), aa, acc[c]);
            else if constexpr (V == 2) acc[c] = min2(add2(bv[c], aa), acc[c]);
            else if constexpr (V == 3) acc[c] = __viaddmin_u16x2(bv[c], aa, acc[c]);
            else acc[c] = min2(__vaddus2(bv[c], aa), acc[c]);
        }
        a = (a + 5u) & 0x3FFFu;
    }
    uint32_t x = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) x ^= acc[c];
    if (x == seed) sink[0] = x;
}


__global__ void fill_u16_kernel(uint16_t* p, size_t n, uint16_t v) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------

void launch_leaf_bfs(const uint8_t* pass, int S, int b, int leaves_x, int n_leaves, MatSet leaves,
                     cudaStream_t st, const int* list) {
    const size_t smem = (size_t)kBfsWarps * leaves.NP * sizeof(uint16_t);
    for (int y0 = 0; y0 < n_leaves; y0 += kMaxGridY) {
        dim3 grid(blocks_for(leaves.NP, kBfsWarps), std::min(kMaxGridY, n_leaves - y0));
        leaf_bfs_kernel<<<grid, kBfsWarps * 32, smem, st>>>(pass, S, b, leaves_x, leaves, list, y0);
    }
}

void launch_node_init(MatSet node, MatSet child, const int* child_ext, int nP, int g, int nodes_x,
                      int child_nodes_x, int n_nodes, cudaStream_t st, const int* list) {
    const size_t chunks = (size_t)node.NP * (node.NP / 8);
    for (int y0 = 0; y0 < n_nodes; y0 += kMaxGridY) {
        dim3 grid(blocks_for(chunks, 256), std::min(kMaxGridY, n_nodes - y0));
        node_init_kernel<<<grid, 256, 0, st>>>(node, child, child_ext, nP, g, nodes_x, child_nodes_x, list, y0);
    }
}

void launch_seams_build(MatSet node, const int* seams, int n_seams, const uint8_t* pass, int S, int side,
                        int nodes_x, int n_nodes, uint8_t* kflag, cudaStream_t st, const int* list,
                        const uint16_t* wts) {
    if (n_seams == 0) return;
    for (int y0 = 0; y0 < n_nodes; y0 += kMaxGridY) {
        dim3 grid(blocks_for(n_seams, 128), std::min(kMaxGridY, n_nodes - y0));
        seams_build_kernel<<<grid, 128, 0, st>>>(node, seams, n_seams, pass, wts, S, side, nodes_x, kflag, list, y0);
    }
}

void launch_leaf_weight_init(const uint8_t* pass, const uint16_t* wts, int S, int b, int leaves_x, int n_leaves,
                             MatSet leaves, uint8_t* kflag, const int* list, cudaStream_t st) {
    constexpr int kWarps = 8;
    for (int y0 = 0; y0 < n_leaves; y0 += kMaxGridY) {
        dim3 grid(blocks_for(leaves.NP, kWarps), std::min(kMaxGridY, n_leaves - y0));
        leaf_weight_init_kernel<<<grid, kWarps * 32, 0, st>>>(pass, wts, S, b, leaves_x, leaves, kflag, list, y0);
    }
}

void launch_compact_pivots(const Slot* S, int n, int NP, int* slot_cnt, cudaStream_t st) {
    if (n == 0) return;
    compact_pivots_kernel<<<n, 256, 0, st>>>(S, NP, slot_cnt);
}

template <int RW, int CP, bool PANEL>
static void launch_gemm_t(const Slot* S, int n, int NP, int round, uint16_t* panel, uint8_t* flags,
                          const uint16_t* tstar, cudaStream_t st) {
    constexpr int MT = 8 * RW, NT = 64 * CP;
    const size_t smem = (size_t)kPivotChunk * (MT + NT) * sizeof(uint16_t);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(closure_gemm_kernel<RW, CP, PANEL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        configured = true;
    }
    dim3 grid(NP / NT, PANEL ? 1 : NP / MT, n);
    closure_gemm_kernel<RW, CP, PANEL><<<grid, 256, smem, st>>>(S, NP, round, panel, flags, tstar);
}

size_t closure_scratch_elems(int NP, int n_active) {
    return (size_t)n_active * kPivotChunk * NP + (size_t)n_active * kPivotChunk * kPivotChunk;
}

void launch_closure_round(const Slot* S, int n, int NP, int round, uint16_t* panel, uint8_t* flags,
                          cudaStream_t st) {
    if (n == 0) return;
    uint16_t* tstar = panel + (size_t)n * kPivotChunk * NP;
    pivot_close_kernel<<<n, 256, 0, st>>>(S, NP, round, tstar);
    // Panel tiles: the widest whose grid still has two CTAs per SM (148 SMs).
    const size_t ctas = (size_t)(NP / 64) * n;
    if (NP >= 256 && ctas >= 4 * 296)
        launch_gemm_t<8, 4, true>(S, n, NP, round, panel, flags, tstar, st);
    else if (NP >= 128 && ctas >= 2 * 296)
        launch_gemm_t<8, 2, true>(S, n, NP, round, panel, flags, tstar, st);
    else
        launch_gemm_t<8, 1, true>(S, n, NP, round, panel, flags, tstar, st);
    if (NP >= 256) launch_gemm_t<16, 4, false>(S, n, NP, round, panel, flags, tstar, st);
    else if (NP >= 128) launch_gemm_t<16, 2, false>(S, n, NP, round, panel, flags, tstar, st);
    else launch_gemm_t<8, 1, false>(S, n, NP, round, panel, flags, tstar, st);
}

void launch_leaf_edges(const Slot* S, int n, const int* edges, int NP, int* task_pivots, cudaStream_t st) {
    if (n == 0) return;
    leaf_edges_kernel<<<n, 32, 0, st>>>(S, edges, NP, task_pivots);
}

void launch_node_child_insert(const Slot* S, int n, const int* child_ext, int nP, int g, int NP, int childNP,
                              cudaStream_t st) {
    for (int z0 = 0; z0 < n; z0 += kMaxGridY) {
        dim3 grid(blocks_for((size_t)nP * nP, 256), g * g, std::min(kMaxGridY, n - z0));
        node_child_insert_kernel<<<grid, 256, 0, st>>>(S + z0, child_ext, nP, g, NP, childNP);
    }
}

void launch_node_seams(const Slot* S, int n, const int* seams, int NP, cudaStream_t st) {
    if (n == 0) return;
    node_seams_kernel<<<n, 32, 0, st>>>(S, seams, NP);
}

void launch_ext_snapshot(const Slot* S, int n, const int* ext, int nExt, int NP, uint16_t* snap, cudaStream_t st) {
    for (int y0 = 0; y0 < n; y0 += kMaxGridY) {
        dim3 grid(blocks_for((size_t)nExt * nExt, 256), std::min(kMaxGridY, n - y0));
        ext_snapshot_kernel<<<grid, 256, 0, st>>>(S + y0, ext, nExt, NP, snap + (size_t)y0 * nExt * nExt);
    }
}

void launch_ext_compare(const Slot* S, int n, const int* ext, int nExt, int NP, const uint16_t* snap,
                        uint8_t* slot_dec, int g, cudaStream_t st, int any_change) {
    for (int y0 = 0; y0 < n; y0 += kMaxGridY) {
        dim3 grid(blocks_for((size_t)nExt * nExt, 256), std::min(kMaxGridY, n - y0));
        ext_compare_kernel<<<grid, 256, 0, st>>>(S + y0, ext, nExt, NP, snap + (size_t)y0 * nExt * nExt,
                                                 slot_dec + y0, g, any_change);
    }
}

void launch_fill_u16(uint16_t* ptr, size_t n, uint16_t value, cudaStream_t st) {
    if (n == 0) return;
    fill_u16_kernel<<<(unsigned)std::min<size_t>(blocks_for(n, 256), 148 * 8), 256, 0, st>>>(ptr, n, value);
}

void launch_gather_block(const uint16_t* mat, int NP, const int* rows, int nr, const int* cols, int nc,
                         uint16_t* out, cudaStream_t st) {
    const size_t n = (size_t)nr * nc;
    if (n == 0) return;
    gather_block_kernel<<<blocks_for(n, 256), 256, 0, st>>>(mat, NP, rows, nr, cols, nc, out);
}

void launch_digest(MatSet M, int count, unsigned long long* out, cudaStream_t st) {
    const size_t rows = (size_t)count * M.n;
    if (rows == 0) return;
    const unsigned grid = (unsigned)std::min<size_t>(rows, 148 * 8);
    digest_kernel<<<grid, 256, 0, st>>>(M, count, out);
}


double measure_minplus_rate(int variant, int sms) {
    const int iters = 4096, threads = 512, blocks = sms * 4;
    uint32_t* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(uint32_t)) != cudaSuccess) return -1.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto launch = [&](int it) {
        switch (variant) {
            case 0: minplus_rate_kernel<0><<<blocks, threads>>>(it, 12345u, sink); break;
            case 1: minplus_rate_kernel<1><<<blocks, threads>>>(it, 12345u, sink); break;
            case 2: minplus_rate_kernel<2><<<blocks, threads>>>(it, 12345u, sink); break;
            case 3: minplus_rate_kernel<3><<<blocks, threads>>>(it, 12345u, sink); break;
            default: minplus_rate_kernel<4><<<blocks, threads>>>(it, 12345u, sink); break;
        }
    };
    launch(64);  // warm-up
    cudaEventRecord(e0);
    launch(iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    return (double)blocks * threads * iters * 16.0 / (ms * 1e-3);
}

}  // namespace hb
