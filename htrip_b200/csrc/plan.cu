// queryAllPairs planning on the device.  plan_query_kernel turns the
// viewpoints (device memory) into the plan the persistent query kernel reads,
// so a query whose inputs are already in HBM needs no host round trip.  It
// writes the plan the host planner (index.cu make_plan) writes for the same
// tile shape, except that each level's finite-port flags start at a fixed
// offset (the capacity of the levels below); batches of several requests, the
// allocation-free entry point and the autotuner keep using the host planner.
//
// Grid: one planning block per hierarchy level (block l-1 plans level l;
// one block when H = 0), then blocks that preset the pair matrix and clear
// the flags.  The levels of a plan are independent once the viewpoints are
// ordered, so every planning block sorts them itself:
//   1. passable viewpoints get the key (Morton code of their leaf, base g^2,
//      level-1 digit least significant) * 2^12 + original index; a bitonic
//      sort orders them (the host's stable sort by Morton code): shuffles for
//      strides below 32, ping-pong shared buffers above;
//   2. block 0: per sorted viewpoint its leaf, cell in leaf and leaf run;
//      original -> sorted; the launch words cleared;
//   3. block l-1: the child groups of level l (runs of one level-(l-1) node);
//      per group its slot run (padded to RW), its project items and its meet
//      base items, the three prefix sums in one pass; the group table, the
//      slot -> viewpoint table, the level-0 table (l = 1), project items and
//      meet items (each base item split over the ports so the level has about
//      296), one slot or item per thread; then the groups and slots of level
//      l+1 for the lift table of level l;
//   4. every planning block files its counts and takes a ticket; the block
//      with the last ticket writes the request's header, the units per phase,
//      the status and the host-mapped record (one 8-byte word: seq << 32 |
//      status << 26 | viewpoints << 13 | largest root child group), from which
//      the host picks its next tile shape.
// Capacities come from the host (PlanLayout, worst cases for k); a plan that
// would not fit sets status 2 and gives the query kernel no work.  No block
// waits for another.
#include "kernels.cuh"

#include <algorithm>
#include <atomic>
#include <cstdint>

namespace hb {

namespace {

constexpr int kPlanMaxThreads = 1024;
constexpr int kPlanMaxK = 4096;
constexpr int kRec = 8;  // ints of a level's record

__device__ __forceinline__ int n_warps() { return blockDim.x >> 5; }

// x / d and x % d for x >= 0, with shifts when d = 2^sh (sh >= 0).
__device__ __forceinline__ int divp(int x, int d, int sh) { return sh >= 0 ? x >> sh : x / d; }
__device__ __forceinline__ int modp(int x, int d, int sh) { return sh >= 0 ? x & (d - 1) : x % d; }

// Exclusive prefix sums of up to three sequences f(i) = {x, y, z}, i in
// [0, n), evaluated once each by the thread that owns i's chunk, into
// a[i], b[i], c[i] (null to skip); returns the totals.  Every thread of the
// block calls it; ends synchronised.
template <class F>
__device__ int3 block_scan3(F f, int n, int* a, int* b, int* c, int* ws) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = n_warps();
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int b0 = min(n, tid * per), b1 = min(n, b0 + per);
    int3 loc = make_int3(0, 0, 0);
    for (int i = b0; i < b1; ++i) {
        const int3 v = f(i);
        if (a) a[i] = v.x;
        if (b) b[i] = v.y;
        if (c) c[i] = v.z;
        loc.x += v.x;
        loc.y += v.y;
        loc.z += v.z;
    }
    int3 inc = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, inc.x, o);
        const int y = __shfl_up_sync(0xffffffffu, inc.y, o);
        const int z = __shfl_up_sync(0xffffffffu, inc.z, o);
        if (lane >= o) {
            inc.x += x;
            inc.y += y;
            inc.z += z;
        }
    }
    if (lane == 31) {
        ws[warp] = inc.x;
        ws[33 + warp] = inc.y;
        ws[66 + warp] = inc.z;
    }
    __syncthreads();
    if (warp == 0) {
        for (int s = 0; s < 3; ++s) {
            const int w = lane < nw ? ws[33 * s + lane] : 0;
            int wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += v;
            }
            if (lane < nw) ws[33 * s + lane] = wi - w;
            if (lane == 31) ws[33 * s + 32] = wi;
        }
    }
    __syncthreads();
    int rx = ws[warp] + inc.x - loc.x, ry = ws[33 + warp] + inc.y - loc.y, rz = ws[66 + warp] + inc.z - loc.z;
    for (int i = b0; i < b1; ++i) {
        if (a) { const int v = a[i]; a[i] = rx; rx += v; }
        if (b) { const int v = b[i]; b[i] = ry; ry += v; }
        if (c) { const int v = c[i]; c[i] = rz; rz += v; }
    }
    const int3 tot = make_int3(ws[32], ws[65], ws[98]);
    __syncthreads();
    return tot;
}

// Largest q in [0, n) with a[q] <= x (a nondecreasing, a[0] <= x).
__device__ __forceinline__ int last_le(const int* a, int n, int x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Preset blocks: M = 0xFF.., flags = 0.
__device__ void plan_fill(const PlanLayout& O, int first) {
    const long nb = gridDim.x - first, b = blockIdx.x - first;
    const long stride = nb * blockDim.x;
    int4* m = reinterpret_cast<int4*>(O.M);
    const long m16 = O.M_bytes / 16;
    const int4 ff = make_int4(-1, -1, -1, -1);
    for (long i = b * blockDim.x + threadIdx.x; i < m16; i += stride) m[i] = ff;
    int4* f = reinterpret_cast<int4*>(O.flags);
    const long f16 = O.flags_bytes / 16;
    const int4 z = make_int4(0, 0, 0, 0);
    for (long i = b * blockDim.x + threadIdx.x; i < f16; i += stride) f[i] = z;
    for (long i = f16 * 16 + b * blockDim.x + threadIdx.x; i < O.flags_bytes; i += stride) O.flags[i] = 0;
}

// Parts per project item of level l: the template's split while the level
// has at most G.split_items items (the host sized the part scratch so).
__device__ __forceinline__ int level_split(const QueryParams& tmpl, const PlanGeom& G, int l, int n_items) {
    const int s = tmpl.lv[l].split;
    return s > 1 && n_items <= G.split_items ? s : 1;
}

__device__ __forceinline__ bool vp_inside(const int32_t* vps, const uint8_t* pf, int i, int S) {
    const int r = vps[2 * i], c = vps[2 * i + 1];  // loaded together with the flag
    return pf[i] && r >= 0 && c >= 0 && r < S && c < S;
}

__device__ __forceinline__ unsigned long long vp_key(const int32_t* vps, const uint8_t* pf, int i, int k,
                                                     const PlanGeom& G) {
    if (i >= k || !vp_inside(vps, pf, i, G.S)) return ~0ull;
    int x = divp(vps[2 * i + 1], G.b, G.b_shift), y = divp(vps[2 * i], G.b, G.b_shift);
    unsigned long long m = 0, mul = 1;
    const unsigned long long g2 = (unsigned long long)G.g * G.g;
    for (int l = 0; l < max(G.H, 1); ++l) {
        m += (unsigned long long)(modp(y, G.g, G.g_shift) * G.g + modp(x, G.g, G.g_shift)) * mul;
        mul *= g2;
        x = divp(x, G.g, G.g_shift);
        y = divp(y, G.g, G.g_shift);
    }
    return (m << 12) | (unsigned long long)i;
}

// Shared working arrays of a planning block (N = sort size).
struct PlanSmem {
    unsigned long long *kb0, *kb1;  // sort buffers
    int *sa, *sb;                   // prefix scratch (alias the sort buffers)
    int *ord, *vtx, *vty, *slot;    // per sorted viewpoint
    int *gstart, *gslot0, *gnode, *gquad, *ghead;  // per group (+1)
};

// Child groups of level l (runs of one level-(l-1) node) among the ns
// sorted viewpoints: gstart[0..ngr] (sa: per viewpoint the number of group
// heads before it), node and quadrant of every group.
__device__ int level_groups(const PlanSmem& W, const PlanGeom& G, int l, int ns, int* ws, int* root_max) {
    const int tid = threadIdx.x, nt = blockDim.x, g = G.g;
    const int gl = G.side[l - 1] / G.b;  // leaves per level-(l-1) node side: g^(l-1)
    const int gsh = G.g_shift >= 0 ? G.g_shift * (l - 1) : -1;
    const int ngr = block_scan3([&](int i) {
        int head = 0;
        if (i < ns)
            head = i == 0 || divp(W.vtx[i], gl, gsh) != divp(W.vtx[i - 1], gl, gsh) ||
                   divp(W.vty[i], gl, gsh) != divp(W.vty[i - 1], gl, gsh);
        return make_int3(head, 0, 0);
    }, ns + 1, W.sa, nullptr, nullptr, ws).x;
    for (int i = tid; i < ns; i += nt)
        if (W.sa[i + 1] != W.sa[i]) W.gstart[W.sa[i]] = i;
    if (tid == 0) W.gstart[ngr] = ns;
    __syncthreads();
    const int nx = G.nodes_x[l];
    for (int q = tid; q < ngr; q += nt) {
        const int s0 = W.gstart[q];
        const int cx = divp(W.vtx[s0], gl, gsh), cy = divp(W.vty[s0], gl, gsh);
        W.gnode[q] = divp(cy, g, G.g_shift) * nx + divp(cx, g, G.g_shift);
        W.gquad[q] = modp(cy, g, G.g_shift) * g + modp(cx, g, G.g_shift);
        if (root_max) atomicMax(root_max, W.gstart[q + 1] - s0);
    }
    __syncthreads();
    return ngr;
}

template <int RW, int NC>
__global__ void __launch_bounds__(kPlanMaxThreads, 1)
plan_query_kernel(const int32_t* __restrict__ vps, const uint8_t* __restrict__ pf, const PlanGeom G,
                  const PlanLayout O, const QueryParams tmpl) {
    const int H = G.H, nlev = max(H, 1);
    if ((int)blockIdx.x >= nlev) {
        plan_fill(O, nlev);
        return;
    }
    extern __shared__ __align__(16) unsigned char plan_smem[];
    __shared__ int ws[99];
    __shared__ int sh_ns, sh_root, sh_last;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int k = O.k, N = O.kpow;  // N: sort size (power of two, >= k)
    const int b = G.b, l = blockIdx.x + 1;
    PlanSmem W;
    W.kb0 = reinterpret_cast<unsigned long long*>(plan_smem);
    W.kb1 = W.kb0 + N;
    W.sa = reinterpret_cast<int*>(plan_smem);
    W.sb = W.sa + N + 2;
    W.ord = reinterpret_cast<int*>(plan_smem + O.sort_bytes);
    W.vtx = W.ord + N;
    W.vty = W.vtx + N;
    W.slot = W.vty + N;
    W.gstart = W.slot + N;
    W.gslot0 = W.gstart + N + 1;
    W.gnode = W.gslot0 + N + 1;
    W.gquad = W.gnode + N;
    W.ghead = W.gquad + N;
    int* plan = O.plan;
    QueryParams* Pq = O.params;
    int* rec = plan + O.o_rec;
    if (tid == 0) {
        sh_ns = 0;
        sh_root = 0;
    }
    // fixed parts of the parameter block; block 0 clears the launch words
    if (tid < 32) {
        const int lane = tid;
        if (l <= H && lane == 0) {
            QueryLevel& lv = Pq->lv[l];
            lv.D = tmpl.lv[l].D;
            lv.NP = tmpl.lv[l].NP;
            lv.nP = tmpl.lv[l].nP;
            lv.ext_inv = tmpl.lv[l].ext_inv;
            lv.store_y = tmpl.lv[l].store_y;
            lv.part = tmpl.lv[l].part;
            lv.ticket = tmpl.lv[l].ticket;
        }
        if (blockIdx.x == 0) {
            for (int i = lane; i < O.words_bytes / 4; i += 32) O.words[i] = 0;
            if (lane == 1) {
                Pq->nExt0 = tmpl.nExt0;
                Pq->cfg = tmpl.cfg;
                Pq->ext0 = tmpl.ext0;
                Pq->leaves = tmpl.leaves;
                for (int j = 0; j <= kMaxQueryLevels; ++j) {
                    Pq->X[j] = tmpl.X[j];
                    Pq->Y[j] = tmpl.Y[j];
                }
                Pq->M = tmpl.M;
                Pq->ctr = tmpl.ctr;
                Pq->out = tmpl.out;
                Pq->work = tmpl.work;
                Pq->dirty = tmpl.dirty;
            }
        }
    }
    // ---- 1. keys and sort
    int ns;
    if (N <= nt) {  // one key per thread; threads from N on hold no key
        unsigned long long key = vp_key(vps, pf, tid, k, G);
        int p = 0;
        for (int size = 2; size <= N; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                unsigned long long other = key;
                if (stride >= 32) {
                    unsigned long long* buf = p ? W.kb1 : W.kb0;
                    if (tid < N) buf[tid] = key;
                    __syncthreads();
                    if (tid < N) other = buf[tid ^ stride];
                    p ^= 1;
                } else if (tid < N) {  // whole warps: N is a multiple of 32
                    other = __shfl_xor_sync(0xffffffffu, key, stride);
                }
                if (tid < N) {
                    const bool keep_min = ((tid & stride) == 0) == ((tid & size) == 0);
                    key = keep_min ? min(key, other) : max(key, other);
                }
            }
        ns = __syncthreads_count(key != ~0ull);
        if (tid < ns) W.ord[tid] = (int)(key & 0xfffu);
    } else {  // N > blockDim: keys in shared memory
        for (int i = tid; i < N; i += nt) W.kb0[i] = vp_key(vps, pf, i, k, G);
        __syncthreads();
        for (int size = 2; size <= N; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int i = tid; i < N; i += nt) {
                    const int j = i ^ stride;
                    if (j > i) {
                        const unsigned long long a = W.kb0[i], c = W.kb0[j];
                        if ((a > c) == ((i & size) == 0)) {
                            W.kb0[i] = c;
                            W.kb0[j] = a;
                        }
                    }
                }
                __syncthreads();
            }
        for (int i = tid; i < N; i += nt)
            if (W.kb0[i] != ~0ull && (i + 1 == N || W.kb0[i + 1] == ~0ull)) sh_ns = i + 1;
        __syncthreads();
        ns = sh_ns;
        for (int i = tid; i < ns; i += nt) W.ord[i] = (int)(W.kb0[i] & 0xfffu);
    }
    // ---- 2. sorted viewpoints (the sort buffers are dead from here on)
    __syncthreads();
    for (int i = tid; i < ns; i += nt) {
        const int o = W.ord[i];
        const int r = vps[2 * o], c = vps[2 * o + 1];
        const int tx = divp(c, b, G.b_shift), ty = divp(r, b, G.b_shift);
        W.vtx[i] = tx;
        W.vty[i] = ty;
        if (blockIdx.x == 0) {
            plan[O.o_inv + o] = i;
            plan[O.o_vp0 + 4 * i] = ty * G.leaves_x + tx;
            plan[O.o_vp0 + 4 * i + 1] = (r - ty * b) * b + (c - tx * b);
        }
    }
    if (blockIdx.x == 0)
        for (int o = tid; o < k; o += nt)
            if (!vp_inside(vps, pf, o, G.S)) plan[O.o_inv + o] = -1;
    __syncthreads();
    if (blockIdx.x == 0) {  // leaf runs
        block_scan3([&](int i) {
            return make_int3(i < ns && (i == 0 || W.vtx[i] != W.vtx[i - 1] || W.vty[i] != W.vty[i - 1]), 0, 0);
        }, ns + 1, W.sa, nullptr, nullptr, ws);
        for (int i = tid; i < ns; i += nt)
            if (W.sa[i + 1] != W.sa[i]) W.gstart[W.sa[i]] = i;
        if (tid == 0) W.gstart[W.sa[ns]] = ns;
        __syncthreads();
        for (int i = tid; i < ns; i += nt) {
            const int h = W.sa[i + 1] - 1;
            plan[O.o_vp0 + 4 * i + 2] = W.gstart[h];
            plan[O.o_vp0 + 4 * i + 3] = W.gstart[h + 1];
        }
        __syncthreads();
    }
    // ---- 3. level l
    int fail = 0, n_items = 0, n_meet = 0, slots = 0;
    if (l <= H) {
        const int nP = G.nP[l], NP = G.NP[l];
        const int ngr = level_groups(W, G, l, ns, ws, l == H ? &sh_root : nullptr);
        // per group: slot run, project items, meet base items.  A group's meet
        // rows start at its node's first slot: s2 - sW is the padded length of
        // the node's earlier groups (at most g^2 - 1 of them).
        const int3 tot = block_scan3([&](int q) {
            if (q >= ngr) return make_int3(0, 0, 0);
            const int cnt = W.gstart[q + 1] - W.gstart[q];
            int h = q, rel = 0;
            while (h > 0 && W.gnode[h - 1] == W.gnode[q]) {
                --h;
                rel += (W.gstart[h + 1] - W.gstart[h] + RW - 1) / RW * RW;
            }
            W.ghead[q] = h;
            const int n_begin = (l == H) ? (W.gquad[q] * nP) / NC * NC : 0;
            const int items = (cnt + RW - 1) / RW * ((NP - n_begin + NC - 1) / NC);
            // base items: per RW-row tile jb, the NC-slot tiles from the node's
            // first slot that reach a later row: ceil((rel + jb + nj - 1) / NC)
            int meet = 0;
            for (int jb = 0; jb < cnt; jb += RW) meet += (rel + jb + min(RW, cnt - jb) - 1 + NC - 1) / NC;
            return make_int3((cnt + RW - 1) / RW * RW, items, meet);
        }, ngr + 1, W.gslot0, W.sa, W.sb, ws);
        slots = tot.x;
        n_items = tot.y;
        const int nbase = tot.z;
        int ks = nbase ? (kPlanTargetItems + nbase - 1) / nbase : 1;
        ks = max(1, min(ks, (nP + 63) / 64));
        const int kstep = ((nP + ks - 1) / ks + 31) / 32 * 32;
        const int nsplit = (nP + kstep - 1) / kstep;
        n_meet = nbase * nsplit;
        fail = ngr > O.cap_groups[l] || slots > O.cap_slots[l] || n_items > O.cap_items[l] ||
               n_meet > O.cap_meet[l];  // uniform: every thread holds the same totals
        if (!fail) {
            int* grp = plan + O.o_groups[l];
            int* s2v = plan + O.o_s2v[l];
            int* l0 = plan + O.o_l0;
            int* lift = l < H ? plan + O.o_lift[l] : nullptr;
            int* items = plan + O.o_items[l];
            int* meet = plan + O.o_meet[l];
            // slot tables, one slot per thread (neighbouring threads store to
            // neighbouring words); the lift table's padding entries are 0
            for (int s = tid; s < slots + NC; s += nt) {
                if (s >= slots) {
                    s2v[s] = -1;
                    continue;
                }
                const int q = last_le(W.gslot0, ngr, s);
                const int idx = s - W.gslot0[q];
                if (idx < W.gstart[q + 1] - W.gstart[q]) {
                    const int i = W.gstart[q] + idx;
                    s2v[s] = i;
                    W.slot[i] = s;
                    if (l == 1) {
                        l0[2 * s] = i;
                        l0[2 * s + 1] = q;
                    }
                } else {
                    s2v[s] = -1;
                    if (l == 1) {
                        l0[2 * s] = -1;
                        l0[2 * s + 1] = -1;
                    }
                    if (lift) {
                        lift[2 * s] = 0;
                        lift[2 * s + 1] = 0;
                    }
                }
            }
            for (int e = tid; e < 5 * ngr; e += nt) {
                const int q = e / 5, f = e - 5 * q;
                grp[e] = f == 0 ? W.gnode[q] : f == 1 ? W.gquad[q] : f == 2 ? W.gslot0[q]
                       : f == 3 ? W.gstart[q + 1] - W.gstart[q] : W.gstart[q];
            }
            for (int w = tid; w < n_items; w += nt) {
                const int q = last_le(W.sa, ngr, w);
                const int e = w - W.sa[q];
                const int n_begin = (l == H) ? (W.gquad[q] * nP) / NC * NC : 0;
                const int ntile = (NP - n_begin + NC - 1) / NC;
                items[3 * w] = q;
                items[3 * w + 1] = (e / ntile) * RW;
                items[3 * w + 2] = n_begin + (e % ntile) * NC;
            }
            for (int bi = tid; bi < nbase; bi += nt) {
                const int q = last_le(W.sb, ngr, bi);
                const int cnt = W.gstart[q + 1] - W.gstart[q], s0 = W.gslot0[q], sW = W.gslot0[W.ghead[q]];
                // the r-th base tile of q in (slot tile t, row tile j) order; the
                // row tiles of slot tile t are the suffix j >= jfirst(t)
                int r = bi - W.sb[q], t = 0, j = 0;
                const int njb = (cnt + RW - 1) / RW, rel = s0 - sW;
                for (;; ++t) {
                    int lo = 0, hi = njb - 1;  // first j with rel + j*RW + nj - 1 > t*NC (the last one is)
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (rel + mid * RW + min(RW, cnt - mid * RW) - 1 > t * NC) hi = mid;
                        else lo = mid + 1;
                    }
                    if (r < njb - lo) {
                        j = lo + r;
                        break;
                    }
                    r -= njb - lo;
                }
                const int jb = j * RW;
                for (int sp = 0; sp < nsplit; ++sp) {
                    const int kb = sp * kstep;
                    int* it = meet + 7 * (bi * nsplit + sp);
                    it[0] = sW + t * NC;
                    it[1] = s0 + jb;
                    it[2] = min(RW, cnt - jb);
                    it[3] = q;
                    it[4] = W.gquad[q] * nP;
                    it[5] = kb;
                    it[6] = min(nP, kb + kstep);
                }
            }
            if (tid == 0) {
                QueryLevel& lv = Pq->lv[l];
                lv.groups = grp;
                lv.flags = O.flags + O.flags_off[l];
                lv.items = items;
                lv.n_items = n_items;
                lv.split = level_split(tmpl, G, l, n_items);
                lv.meet = meet;
                lv.n_meet = n_meet;
                lv.s2v = s2v;
                lv.lift = lift;
            }
            if (lift) {  // level l slot -> {level-(l+1) slot, level-(l+1) group}
                __syncthreads();
                const int ngr2 = level_groups(W, G, l + 1, ns, ws, nullptr);
                block_scan3([&](int q) {
                    return make_int3(q < ngr2 ? (W.gstart[q + 1] - W.gstart[q] + RW - 1) / RW * RW : 0, 0, 0);
                }, ngr2 + 1, W.gslot0, nullptr, nullptr, ws);
                for (int i = tid; i < ns; i += nt) {
                    const int q2 = W.sa[i + 1] - 1;
                    lift[2 * W.slot[i]] = W.gslot0[q2] + (i - W.gstart[q2]);
                    lift[2 * W.slot[i] + 1] = q2;
                }
            }
        }
    }
    // ---- 4. file this block's counts; the last block assembles the request
    __syncthreads();
    if (tid == 0) {
        int* r = rec + kRec * blockIdx.x;
        r[0] = fail;
        r[1] = n_items;
        r[2] = n_meet;
        r[3] = slots;
        r[4] = sh_root;
        __threadfence();
        const unsigned ticket = atomicAdd(O.ticket, 1u);
        sh_last = ticket - O.ticket_base == (unsigned)(nlev - 1);
    }
    __syncthreads();
    if (!sh_last || tid >= 32) return;
    __threadfence();
    // warp 0 of the last block: lane c reads level c+1's record
    const int lane = tid;
    const volatile int* vr = rec + kRec * lane;
    const bool own = lane < nlev;
    const int r_fail = own ? vr[0] : 0, r_items = own ? vr[1] : 0, r_meet = own ? vr[2] : 0;
    int r_slots = own ? vr[3] : 0;
    const int r_root = own ? vr[4] : 0;
    const bool any_fail = __any_sync(0xffffffffu, r_fail != 0);
    for (int o = 16; o > 0; o >>= 1) r_slots = max(r_slots, __shfl_xor_sync(0xffffffffu, r_slots, o));
    const int ldv = (max(ns, r_slots) + 256 + 7) / 8 * 8;
    const bool bad = any_fail || ldv > O.cap_ldv;
    const int n_l0 = H >= 1 ? __shfl_sync(0xffffffffu, own ? vr[3] : 0, 0) : 0;
    const int root = H >= 1 ? __shfl_sync(0xffffffffu, r_root, H - 1) : ns;
    // phase t: project items of level t (lane t-1), meet items of level t-1 (lane t-2)
    const int items_l = __shfl_sync(0xffffffffu, r_items, max(lane - 1, 0));
    const int items_t = items_l * (lane >= 1 && lane <= H ? level_split(tmpl, G, lane, items_l) : 1);
    const int meet_t = __shfl_sync(0xffffffffu, r_meet, max(lane - 2, 0));
    const int n_phases = H + 3;
    if (lane < n_phases) {
        const int t = lane;
        long u;
        if (t == 0)
            u = ((long)n_l0 * G.nExt0 + kQueryL0Chunk - 1) / kQueryL0Chunk + (ns + kQueryThreads - 1) / kQueryThreads;
        else if (t <= H + 1)
            u = (t <= H ? items_t : 0) + (t >= 2 ? meet_t : 0);
        else
            u = ((long)k * k + kQueryFinChunk - 1) / kQueryFinChunk;
        O.unit_pre[2 * t] = 0;
        O.unit_pre[2 * t + 1] = bad ? 0 : (int)u;  // a plan that did not fit: no work at all
    }
    if (lane == 0) {
        Pq->H = H;
        Pq->k = k;
        Pq->ns = ns;
        Pq->ldv = ldv;
        Pq->ldm = max(8, (ns + 7) / 8 * 8);
        Pq->n_l0_slots = n_l0;
        Pq->vp0 = plan + O.o_vp0;
        Pq->inv = plan + O.o_inv;
        Pq->l0 = plan + O.o_l0;
        if (bad) O.words[0] = 2;
        // host record in one 8-byte store: seq | root (13 bits) | ns (13 bits) | status (2 bits)
        if (O.info)
            *reinterpret_cast<volatile unsigned long long*>(O.info) =
                ((unsigned long long)(unsigned)O.seq << 32) |
                (unsigned)(root | ns << 13 | (bad ? 2 : 0) << 26);
    }
}

using PlanKernel = void (*)(const int32_t*, const uint8_t*, const PlanGeom, const PlanLayout, const QueryParams);

PlanKernel plan_kernel_for(int RW, int NC) {
    if (RW == 8 && NC == 64) return plan_query_kernel<8, 64>;
    if (RW == 8 && NC == 128) return plan_query_kernel<8, 128>;
    if (RW == 16 && NC == 128) return plan_query_kernel<16, 128>;
    if (RW == 8 && NC == 256) return plan_query_kernel<8, 256>;
    return nullptr;
}

}  // namespace

int plan_max_k() { return kPlanMaxK; }

int plan_kpow(int k) {
    int p = 128;
    while (p < k) p <<= 1;
    return p;
}

int plan_threads(int) { return kPlanMaxThreads; }

size_t plan_sort_bytes(int kpow) {
    // two ping-pong key buffers for the register sort, one for the shared
    // sort; at least the two prefix scratch arrays that alias them
    const size_t keys = (kpow <= kPlanMaxThreads ? 16 : 8) * (size_t)kpow;
    return std::max(keys, (2 * (size_t)kpow + 4) * sizeof(int));
}

size_t plan_smem_bytes(int kpow) { return plan_sort_bytes(kpow) + (9 * (size_t)kpow + 2) * sizeof(int); }

int plan_record_ints() { return kRec * (kMaxQueryLevels + 1); }

cudaError_t launch_plan_query(const int32_t* vps, const uint8_t* pf, const PlanGeom& G, const PlanLayout& O,
                              const QueryParams& tmpl, int fill_blocks, cudaStream_t st) {
    const PlanKernel kern = plan_kernel_for(G.RW, G.NC);
    if (!kern || O.kpow != plan_kpow(O.k) || O.sort_bytes != plan_sort_bytes(O.kpow) || O.k > kPlanMaxK ||
        G.H > kMaxQueryLevels)
        return cudaErrorInvalidValue;
    const size_t smem = plan_smem_bytes(O.kpow);
    if (smem > 48 * 1024) {
        // once per device and tile shape: the largest dynamic shared memory any k needs
        static std::atomic<unsigned> configured[64];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
        const unsigned bit = 1u << (G.RW == 16 ? 2 : G.NC == 64 ? 0 : G.NC == 128 ? 1 : 3);
        if (!(configured[dev].load() & bit)) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan_smem_bytes(kPlanMaxK));
            if (e != cudaSuccess) return e;
            configured[dev].fetch_or(bit);
        }
    }
    kern<<<std::max(G.H, 1) + fill_blocks, plan_threads(O.kpow), smem, st>>>(vps, pf, G, O, tmpl);
    return cudaGetLastError();
}

}  // namespace hb
