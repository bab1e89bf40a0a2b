// Kernel launch wrappers (htrip_b200/csrc/kernels.cu).  All launches are
// asynchronous on the given stream; the caller checks cudaGetLastError.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace hb {

// One square u16 matrix family: `count` matrices of logical order n padded
// to NP (multiple of 64), matrix m at base + m*NP*NP, row-major.
struct MatSet {
    uint16_t* base;
    int n;
    int NP;
};

constexpr int kPivotChunk = 64;   // pivots closed per round (B)
constexpr int kFlagTile = 64;     // column granularity of panel "finite" flags

// --- build ------------------------------------------------------------------
// Leaf APSP by bit-parallel BFS (reference LeafTile::recomputeFromGrid,
// leaf_tile.cpp:96-153).  pass: S*S bytes, 1 = Free.
// With `list`, the n_leaves leaves list[0..n_leaves) instead of 0..n_leaves.
void launch_leaf_bfs(const uint8_t* pass, int S, int b, int leaves_x, int n_leaves, MatSet leaves,
                     cudaStream_t st, const int* list = nullptr);

// Internal-node initial D_U: block diagonal of child summaries, INF
// elsewhere (internal_node.cpp:98-145).  child_ext: the child level's
// port -> matrix-index table (nP entries).
void launch_node_init(MatSet node, MatSet child, const int* child_ext, int nP, int g, int nodes_x,
                      int child_nodes_x, int n_nodes, cudaStream_t st, const int* list = nullptr);

// Seam edges of the build (internal_node.cpp:155-173): seams = 6 ints per
// candidate {u, v, ur, uc, vr, vc} (node-relative coordinates).
// wts (optional): per-cell traversal weights (S x S); a seam gets the edge
// weight w(u, v) = max(1, (w_u + w_v) / 2) (GridMap::edgeWeight), else 1.
void launch_seams_build(MatSet node, const int* seams, int n_seams, const uint8_t* pass, int S,
                        int side, int nodes_x, int n_nodes, uint8_t* kflag, cudaStream_t st,
                        const int* list = nullptr, const uint16_t* wts = nullptr);

// Weighted leaves (the reference's Dijkstra leaf build): D = the tile's
// weighted adjacency with a zero diagonal, pivot flags = its passable cells;
// a closure over those pivots then gives the leaf's shortest-path matrix.
void launch_leaf_weight_init(const uint8_t* pass, const uint16_t* wts, int S, int b, int leaves_x, int n_leaves,
                             MatSet leaves, uint8_t* kflag, const int* list, cudaStream_t st);

// One matrix of an update launch (any index, any map size: the launch's
// matrices share b, g and level, hence order, padding and port tables).
struct Slot {
    uint16_t* mat;              // the matrix (NP x NP)
    uint8_t* kflag;             // its pivot flags (NP)
    int* klist;                 // its pivot list (NP)
    int* kcnt;                  // its pivot count
    uint8_t* dec;               // its summary-decreased flag
    const uint16_t* child_mat;  // node slots: the child level's matrices (null for leaves)
    uint8_t* child_dec;         // node slots: the child level's decrease flags (null for leaves)
    int node, nodes_x, child_nodes_x;
    int list_begin, list_end;   // the slot's range of the launch's edge / seam list
    int task;                   // the slot's opening task within the launch
    int root;                   // 1: the index's root (no summary above it)
};

// --- closure over pivot sets -------------------------------------------------
// Compact every slot's pivot flags into its sorted list (clears the flags);
// slot_cnt (optional) receives the counts in slot order as well.
void launch_compact_pivots(const Slot* S, int n, int NP, int* slot_cnt, cudaStream_t st);

// One round of the blocked pivot-set Kleene closure of every slot: pivots
// klist[round*B .. round*B+B).  panel: closure_scratch_elems(NP, n) u16 of
// scratch; flags: n * NP / kFlagTile bytes.
size_t closure_scratch_elems(int NP, int n_active);
void launch_closure_round(const Slot* S, int n, int NP, int round, uint16_t* panel, uint8_t* flags,
                          cudaStream_t st);

// --- incremental updates -----------------------------------------------------
// Insert opened in-leaf edges (leaf_tile.cpp:311-330): slot s's (u, v, w)
// triples are edges[3*list_begin .. 3*list_end); marks pivot flags and adds
// the new pivots to task_pivots[task].
void launch_leaf_edges(const Slot* S, int n, const int* edges, int NP, int* task_pivots, cudaStream_t st);

// Child-summary decreases into parent D_U (internal_node.cpp:343-353): for
// each slot and each child whose decrease flag is set, insert every child
// summary entry smaller than the parent's and mark both endpoints.
void launch_node_child_insert(const Slot* S, int n, const int* child_ext, int nP, int g, int NP, int childNP,
                              cudaStream_t st);

// Seam edges of an update (internal_node.cpp:356-365): slot s's (u, v, w)
// V_U triples are seams[3*list_begin .. 3*list_end).
void launch_node_seams(const Slot* S, int n, const int* seams, int NP, cudaStream_t st);

// Snapshot / compare of the non-root slots' exterior block (summary S or
// S_U): snap holds nExt*nExt entries per slot; compare sets *dec and
// slot_dec[slot] when any entry decreased (refreshBoundarySummary,
// leaf_tile.cpp:253-273, internal_node.cpp:415-433) and clears the node
// slots' children's decrease flags.  With any_change != 0 (rebuilds) it only
// sets slot_dec[slot] when any exterior entry differs from the snapshot.
void launch_ext_snapshot(const Slot* S, int n, const int* ext, int nExt, int NP, uint16_t* snap, cudaStream_t st);
void launch_ext_compare(const Slot* S, int n, const int* ext, int nExt, int NP, const uint16_t* snap,
                        uint8_t* slot_dec, int g, cudaStream_t st, int any_change = 0);

// --- device-driven openings (open.cu) -----------------------------------------
// One onBatchCellsOpened call (or several, on indexes of equal b and g) as ONE
// cooperative persistent kernel: the level loop, the work list of every level
// and the closure rounds run on the device, phases separated by bounded grid
// barriers; the host uploads the call's cell-derived lists once and reads the
// statistics back once.
constexpr int kOpenMaxLevels = 17;  // H <= 16
constexpr int kOpenB = 64;          // pivots closed per round

// Geometry of one level, shared by every index of a launch (equal b and g).
struct OpenLevelGeom {
    int NP, n, nExt, nP;       // padded / logical order, exterior ports, ports per child
    const uint8_t* isext;      // [NP] 1 = exterior port (leaf perimeter cell / node exterior port)
    const int* child_ext;      // levels >= 1: the child level's port -> matrix index (nP entries)
    int childNP;               // levels >= 1: the child level's padded order
};

// One index ("task") of a launch, per level.
struct OpenTaskLevel {
    uint16_t* mat;             // matrices (NP x NP each)
    uint8_t* kflag;            // pivot flags [node][NP] (zero outside a call)
    int* klist;                // pivot lists [node][NP]
    int* kcnt;                 // pivot counts [node]
    uint32_t* dstamp;          // [node] stamp of the call that decreased the node's exterior block
    uint32_t* mstamp;          // [node] stamp of the call that listed the node
    int nodes_x;
};

// Results of one task, written by the kernel (the host zeroes them first,
// except n_dirty, which starts at the task's number of seam-only nodes).
struct OpenTaskOut {
    int new_pivots;            // leaf pivots set by the call (LastBatchStats::n_pivots)
    int n_dirty;               // listed nodes of levels >= 1 (LastBatchStats::n_dirty_ancestors)
    int level[kOpenMaxLevels][3];  // per level: matrices, sum of pivot counts, largest pivot count
    unsigned long long ops, bytes; // algorithmic work: n^2 k ops, 4 n^2 + 4 k n bytes per matrix
};

struct OpenTask {
    int H;
    int g;
    uint32_t stamp;            // this call's stamp (never 0)
    OpenTaskOut* out;
    OpenTaskLevel lv[kOpenMaxLevels];
};

// What the closure phases of a slot need, in one record written by the slot's
// compaction: its matrix, its pivot list and count, its task and node.
struct OpenSlotRec {
    uint16_t* mat;
    const int* klist;
    int kcnt, task, node;
    int ready;  // 1 once the compaction wrote the record (zero at launch)
};

// Work list entry: {task, node, list_begin, list_end}; the list is the slot's
// range of (u, v, w) triples (level 0: opened in-leaf edges; above: seams).
struct OpenLaunch {
    int n_tasks, maxH, g;
    const OpenTask* tasks;
    OpenLevelGeom geo[kOpenMaxLevels];
    int4* slots[kOpenMaxLevels];   // per level; levels >= 1 start with the seam nodes
    int* count;                    // [kOpenMaxLevels] listed slots per level (grows during the call)
    int4* dchild[kOpenMaxLevels];  // levels >= 1: {task, child, node, quad} of every child whose
                                   // summary decreased (capacity: the child level's cap)
    int* dcount;                   // [kOpenMaxLevels] entries of dchild
    OpenSlotRec* rec[kOpenMaxLevels];  // per level and slot (capacity: the level's cap)
    int cap[kOpenMaxLevels];       // capacity of each level's list
    int n_seam[kOpenMaxLevels];    // seam nodes at the head of each level's list (stamped first)
    int* maxk;                     // [kOpenMaxLevels] largest pivot count per level
    const int* triples;            // (u, v, w)
    uint16_t* panel;               // two buffers (rounds alternate) of, per slot, kOpenB x NP: the
                                   // round's closed pivot rows
    uint8_t* pflags;               // two buffers of, per slot, NP / 64 flags: 64-column blocks of
                                   // the panel holding a finite value
    size_t panel_stride;           // elements between the two panel buffers
    size_t pflag_stride;           // bytes between the two flag buffers
    int* status;                   // 0 ok, 1 a bounded barrier wait timed out, 2 a list overflowed
    unsigned* bar;                 // {arrival count, unit tickets of even / odd phases}
    unsigned* sm;                  // {first CTAs, other CTAs, SM id overflow, per-SM arrivals
                                   //  [kOpenSmSlots]}: the CTAs' SM-aware order (zero at launch)
    unsigned long long* trace;     // or null: [0] start, then one stamp per phase (max kOpenTrace)
};
constexpr int kOpenTrace = 1024;
constexpr int kOpenSmSlots = 256;

// An index's per-level "listed by opening call" stamps, for the dirty
// flags of an incremental query (launch_incremental_dirty): viewpoint j
// (sorted order, leaf vp0[4 j]) gets dirty[j] = 1 + the lowest level whose
// matrix on its leaf-to-root chain carries a stamp newer than `seen` (0: none);
// *n_dirty counts the viewpoints with one.
struct IncrementalChain {
    int H, g, leaves_x;
    const uint32_t* mstamp[kOpenMaxLevels];
    int nodes_x[kOpenMaxLevels];
};
void launch_incremental_dirty(const int* vp0, int ns, const IncrementalChain& C, unsigned seen, uint8_t* dirty,
                              int* n_dirty, cudaStream_t st);

// Shared memory and grid of the launch on `device`; the launch itself.
size_t open_smem_bytes();
int open_grid_blocks(int device);
cudaError_t launch_open(const OpenLaunch& L, int grid, cudaStream_t st);

// --- query (query.cu) -------------------------------------------------------
constexpr int kMaxQueryLevels = 16;
constexpr int kNumQueryConfigs = 4;

// Warp tile of a query work item: RW viewpoint rows x NCOL columns.
struct QueryTile {
    int RW;
    int NCOL;
};
QueryTile query_config_tile(int cfg);
int query_default_config(int NP, int max_group);

struct QueryLevel {
    const uint16_t* D;      // level matrices (NP x NP each)
    int NP, nP;
    const int* ext_inv;     // column -> exterior port index or -1 (NP)
    const int* groups;      // 5 ints per child group {node, quad, slot0, cnt, sorted0}
    uint8_t* flags;         // [group][nP] finite-port flags of X_{l-1}
    const int* items;       // project items {group, m0, n0}
    int n_items;
    const int* meet;        // meet items {i0, j0, nj, group, coloff, kb, ke}
    int n_meet;
    const int* s2v;         // level-l slot -> sorted viewpoint or -1
    const int* lift;        // level-l slot -> {level-(l+1) slot, level-(l+1) group}
    int store_y;
    int split;              // >= 1: every project item runs as `split` units, each over one
                            // part of its compacted port list
    uint32_t* part;         // split > 1: partial tiles [item][part][RW * NC / 2 words]
    unsigned* ticket;       // split > 1: parts of each item done, cleared before the launch
};

// One queryAllPairs request of a launch.
struct QueryParams {
    int H, k, ns, ldv, ldm, n_l0_slots, nExt0, cfg;
    const int* vp0;         // per sorted viewpoint {leaf, u, leaf-run start, leaf-run end}
    const int* inv;         // original index -> sorted index or -1
    const int* l0;          // per level-1 slot {sorted index or -1, level-1 group}
    const int* ext0;        // leaf port -> cell
    MatSet leaves;
    uint16_t* X[kMaxQueryLevels + 1];  // port vectors X_l, l < H ([exterior port of level l][ldv])
    uint16_t* Y[kMaxQueryLevels + 1];  // projections Yt_l, l >= 1 ([column of level l][ldv])
    uint32_t* M;            // sorted-order pair matrix (ldm), preset to 0xFFFFFFFF
    uint16_t* out;          // k x k result
    unsigned* ctr;          // completion counters of the dataflow launch, cleared before it
                            // (query_counter_words): [0] level-0 gather units, [1] project,
                            // meet and same-leaf pair units, [2] root project items,
                            // [4 + l*k + g] rows x column tiles of level-(l-1) project items
                            // done for level-l group g (its target: cnt x column tiles)
    QueryLevel lv[kMaxQueryLevels + 1];
    unsigned long long* work;  // or null: [0] tile entries updated (operand rows streamed x
                               // tile rows x tile columns), [1] operand rows streamed,
                               // [2] operand rows skipped (no finite value in the tile)
    const uint8_t* dirty;      // or null (every viewpoint): per sorted viewpoint, 0 = no node
                               // of its leaf-to-root chain changed, else 1 + the lowest level
                               // whose node changed.  A unit of level l whose rows and columns
                               // are all clean at l (no change at levels <= l) skips its work
                               // (an incremental refresh: the launch's X / Y / flags / M still
                               // hold the previous launch's values for them)
};

// Words of a request's completion counters.
inline size_t query_counter_words(int H, int k) { return 4 + (size_t)(H + 1) * (size_t)(k > 0 ? k : 1); }

// CTA work units of a request in phase t of the launch (host and device
// agree on these numbers):
//   t = 0          level-0 port gathers in chunks of kQueryL0Chunk, then
//                  same-leaf pair rows in chunks of kQueryThreads
//   1 <= t <= H+1  project items of level t (t <= H; `split` units per
//                  item, its parts in order), then meet items of level t-1
//                  (t >= 2)
//   t = H+2        output chunks of kQueryFinChunk entries
#ifndef HB_QUERY_THREADS
#define HB_QUERY_THREADS 256
#endif
constexpr int kQueryThreads = HB_QUERY_THREADS;
constexpr int kQueryL0Chunk = 512;
constexpr int kQueryFinChunk = 1024;

// A launch over n_req requests (any mix of indexes and k on one device).
struct QueryLaunch {
    int n_req;
    int n_phases;              // max over requests of H + 3
    const QueryParams* req;    // device array of n_req requests
    const int* unit_pre;       // [n_phases][n_req + 1]: exclusive prefix of units
    int* status;               // 0 ok, 1 a bounded wait (counter or grid barrier) timed out
    unsigned* bar;             // grid barrier {count, generation}; dataflow: bar[0] is the
                               // ticket that hands out the units
    unsigned long long* trace; // [0, n_phases]: phase starts as CTA 0 sees them (dataflow: [0]
                               // the start, [t + 1] the latest end of a unit of phase t); then
                               // from [kMaxQueryPhases + 1 + t]: the latest end of work of
                               // phase t over all CTAs; or null
    int dataflow;              // 1: no grid barrier - the CTAs take the units of all phases
                               // in ascending order (ticket bar[0]) and each unit first waits
                               // (bounded) for the units whose results it reads
                               // (QueryParams::ctr); 0: phases separated by grid barriers
};
constexpr int kMaxQueryPhases = kMaxQueryLevels + 3;

// Device-side planning of one request (plan.cu): the index's shape and the
// tile of the launch ...
struct PlanGeom {
    int H, g, b, S, leaves_x, RW, NC, nExt0;
    int g_shift, b_shift;              // log2 of g / b when a power of two, else -1
    int side[kMaxQueryLevels + 1];     // node side in cells per level
    int nodes_x[kMaxQueryLevels + 1];  // nodes per row per level
    int nP[kMaxQueryLevels + 1], NP[kMaxQueryLevels + 1];
    int split_items;                   // a level whose template split is > 1 runs split only
                                       // with at most this many project items
};
// ... and where the plan goes: int offsets into `plan` with their capacities
// (worst cases for k viewpoints), each level's flag offset, the request's
// parameter block and unit prefix, the launch words to clear, the presets,
// the ticket counter (ticket_base = its value before this launch; it gains
// max(H, 1) per launch) and an optional host-mapped 8-byte record
// seq << 32 | status << 26 | viewpoints << 13 | largest root child group.
struct PlanLayout {
    int k, kpow;            // kpow = plan_kpow(k): the sort size
    size_t sort_bytes;      // plan_sort_bytes(kpow)
    int* plan;
    int o_vp0, o_inv, o_l0, o_rec;
    long long flags_off[kMaxQueryLevels + 1];
    unsigned* ticket;
    unsigned ticket_base;
    int o_groups[kMaxQueryLevels + 1], o_items[kMaxQueryLevels + 1], o_meet[kMaxQueryLevels + 1];
    int o_s2v[kMaxQueryLevels + 1], o_lift[kMaxQueryLevels + 1];
    int cap_groups[kMaxQueryLevels + 1], cap_slots[kMaxQueryLevels + 1];
    int cap_items[kMaxQueryLevels + 1], cap_meet[kMaxQueryLevels + 1];
    int cap_ldv;
    QueryParams* params;
    int* unit_pre;          // [H + 3][2]
    int* words;             // launch words (status, grid barrier, trace), cleared
    int words_bytes;
    uint32_t* M;            // pair matrix, preset to 0xFF bytes
    long long M_bytes;      // multiple of 16
    uint8_t* flags;         // finite-port flags, cleared
    long long flags_bytes;
    int* info;
    int seq;
};
int plan_max_k();                  // largest k the device planner takes
int plan_kpow(int k);              // power of two >= max(k, 128)
int plan_threads(int kpow);        // threads of a planning block
size_t plan_sort_bytes(int kpow);  // shared bytes of the sort buffers
size_t plan_smem_bytes(int kpow);  // dynamic shared bytes of the planner
int plan_record_ints();            // ints of the per-level records (o_rec)
constexpr int kPlanTargetItems = 296;
// One launch: max(H, 1) planning blocks, then fill_blocks that preset M and
// the flags.
cudaError_t launch_plan_query(const int32_t* vps, const uint8_t* pf, const PlanGeom& G, const PlanLayout& O,
                              const QueryParams& tmpl, int fill_blocks, cudaStream_t st);

// Cooperative launch of the persistent query kernel on `grid` blocks.
int query_grid_blocks(int device);
int query_max_ports();  // largest per-child port count the query kernel handles
// Runs a 4-CTA launch whose grid barrier can never complete (it expects a
// fifth CTA) with a short poll limit: *status is the status word the
// timeout sets (1), *returned the number of CTAs that returned (4).
cudaError_t barrier_timeout_selftest(int* status, int* returned, float* ms);
cudaError_t wait_timeout_selftest(int* status, int* returned, float* ms);
cudaError_t launch_query(const QueryLaunch& L, int cfg, int grid, cudaStream_t st);

// *out += canonical checksum of the first `count` matrices of M (logical
// entries only): sum of splitmix64(((m*n + i)*n + j) << 16 | D[i][j]).
void launch_digest(MatSet M, int count, unsigned long long* out, cudaStream_t st);

// Entries per second of the register-only packed-u16 min-plus update
// (variant 0..3, see minplus_rate_kernel) on `sms` SMs x 4 CTAs; -1 on error.
double measure_minplus_rate(int variant, int sms);

// ptr[0 .. n) = value.
void launch_fill_u16(uint16_t* ptr, size_t n, uint16_t value, cudaStream_t st);

// Gather an exterior block (S / S_U / child_to_ext) of one matrix to dense.
void launch_gather_block(const uint16_t* mat, int NP, const int* rows, int nr, const int* cols, int nc,
                         uint16_t* out, cudaStream_t st);

}  // namespace hb
