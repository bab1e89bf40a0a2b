/*
 * htrip_b200 C ABI: B200-resident HTRIP min-plus hierarchy.
 *
 * The reference (ozaslan/htrip) has no C ABI: its boundary is the C++ class
 * htrip::MinPlusOracle (include/htrip/minplus_oracle.hpp).  Each entry point
 * below replaces one member of that class; the C++ drop-in in
 * include/htrip/minplus_oracle.hpp of this repository calls exactly these.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Unless a name ends in _dev, every array
 *    argument is HOST memory; the call copies it to / from the device itself.
 *  - Cells and viewpoints are int32 pairs (r, c), row-major "rc" arrays.
 *  - Grids are uint8 CellState arrays, rows*cols, row-major:
 *      0 Unknown, 1 Free, 2 Obstacle   (reference include/htrip/types.hpp:100)
 *    Only Free is passable (reference grid_map.hpp:142).
 *  - Distances are uint16 with HTRIP_INF = 60000 for "unreachable".
 *  - Every call returns an htrip_status (0 = ok).  A failed call leaves the
 *    index as it was before the call, except HTRIP_ERR_CUDA, after which the
 *    handle must be destroyed.
 *  - A handle is not thread-safe; distinct handles may be used concurrently
 *    (each owns a CUDA stream).  Calls are synchronous on return.
 */
#ifndef HTRIP_B200_H
#define HTRIP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HTRIP_INF 60000

typedef enum {
    HTRIP_OK = 0,
    HTRIP_ERR_INVALID = 1,     /* bad argument / invalid HierarchyConfig        */
    HTRIP_ERR_NOT_BUILT = 2,   /* update or query before a successful build    */
    HTRIP_ERR_OOM = 3,         /* device allocation failed (index unchanged)   */
    HTRIP_ERR_UNSUPPORTED = 4, /* e.g. tile side outside [2, 32]               */
    HTRIP_ERR_CUDA = 5,        /* CUDA runtime error; destroy the handle       */
    HTRIP_ERR_NO_DEVICE = 6    /* no CUDA device / extension unusable          */
} htrip_status;

typedef struct htrip_index htrip_index; /* opaque */

typedef struct {
    int32_t tile_size_b; /* leaf side b                  (types.hpp:200) */
    int32_t group;       /* g = group_w = group_h        (types.hpp:201-202) */
} htrip_config;

typedef struct {
    int32_t n_touched_leaves;  /* MinPlusOracle::LastBatchStats (minplus_oracle.hpp:251-256) */
    int32_t n_dirty_ancestors;
    int32_t n_pivots;
} htrip_batch_stats;

/* Last error message of the calling thread (static storage). */
const char* htrip_last_error(void);

/* explicit MinPlusOracle(HierarchyConfig)      minplus_oracle.hpp:59
 * `device` selects the CUDA device.  Config validity is checked at build,
 * as in the reference (HierarchyConfig::isValid, types.hpp:221). */
htrip_status htrip_create(htrip_config cfg, int device, htrip_index** out);

/* ~MinPlusOracle                                                         */
htrip_status htrip_destroy(htrip_index* h);

/* MinPlusOracle copy constructor (bench_update_latency.cpp:178,186):
 * deep device-side clone of the whole index.                             */
htrip_status htrip_clone(const htrip_index* h, htrip_index** out);

/* bool build(const GridMap&)                   minplus_oracle.hpp:78
 * observed: rows*cols CellState bytes.  Returns HTRIP_ERR_INVALID where the
 * reference returns false (invalid config, rows or cols <= 0).           */
htrip_status htrip_build(htrip_index* h, const uint8_t* observed, int32_t rows, int32_t cols);

/* void onBatchCellsOpened(cells, grid)         minplus_oracle.hpp:171
 * The caller has already written the cells as Free into `observed`
 * (the grid it passes is read for the cells' neighbours only).           */
htrip_status htrip_open_cells(htrip_index* h, const int32_t* rc, int32_t n,
                              const uint8_t* observed, int32_t rows, int32_t cols);

/* void onCellOpened(Point, grid)               minplus_oracle.hpp:109
 * Same index state as htrip_open_cells with one cell; like the reference it
 * leaves last_batch_stats untouched.                                      */
htrip_status htrip_open_cell(htrip_index* h, int32_t r, int32_t c,
                             const uint8_t* observed, int32_t rows, int32_t cols);

/* void onCellBlocked(Point, const GridMap&)    minplus_oracle.hpp:123
 * The caller has already made the cell non-Free in `observed`.  Its leaf is
 * rebuilt from the grid and every ancestor from its children and seams, up
 * to the root (distances may grow: a non-monotone update).  Cells outside
 * the index are ignored.                                                  */
htrip_status htrip_cell_blocked(htrip_index* h, int32_t r, int32_t c, const uint8_t* observed, int32_t rows,
                                int32_t cols);

/* void onBatchLeavesChanged(const std::vector<int>& leaves, const GridMap&)
 *                                              minplus_oracle.hpp:157
 * Rebuilds the listed leaves (row-major leaf indices; others ignored) from
 * the grid and their ancestors, each dirty ancestor once per level.       */
htrip_status htrip_leaves_changed(htrip_index* h, const int32_t* leaves, int32_t n, const uint8_t* observed,
                                  int32_t rows, int32_t cols);

/* GridMap::weights                             grid_map.hpp:51-56, 297-303
 * The per-cell traversal weights (rows x cols, uint16; NULL: every weight
 * is 1) that build, liftRoot, openings and rebuilds use from now on: an
 * edge between adjacent passable cells costs max(1, (w_u + w_v) / 2), INF
 * when either weight is INF or more (GridMap::edgeWeight, :327-334), and a
 * leaf holding a passable cell of weight != 1 is built as the reference's
 * Dijkstra leaf build does.  Set them before htrip_build; on a built index
 * this refreshes the device copy only (the matrices are not recomputed).  */
htrip_status htrip_set_cell_weights(htrip_index* h, const uint16_t* weights, int32_t rows, int32_t cols);

/* void onCellWeightChanged(Point p, dist_t new_weight, GridMap&)
 *                                              minplus_oracle.hpp:132
 * Sets cell (r, c)'s weight (the library's copy; the caller's grid keeps its
 * own) and rebuilds its leaf and every ancestor; nothing when the cell is
 * outside the grid or its weight is already new_weight (an obstacle's
 * weight is INF).                                                          */
htrip_status htrip_cell_weight_changed(htrip_index* h, int32_t r, int32_t c, uint16_t new_weight,
                                       const uint8_t* observed, int32_t rows, int32_t cols);

/* void onTileWeightsChanged(int tx, int ty, cell_weights, GridMap&)
 *                                              minplus_oracle.hpp:144
 * Sets the weights of the n cells rc[2i], rc[2i+1] to weights[i] (cells
 * outside the grid skipped), then rebuilds leaf (tx, ty) once and every
 * ancestor; nothing when (tx, ty) is not a leaf.                           */
htrip_status htrip_tile_weights_changed(htrip_index* h, int32_t tx, int32_t ty, const int32_t* rc,
                                        const uint16_t* weights, int32_t n, const uint8_t* observed, int32_t rows,
                                        int32_t cols);

/* void liftRoot(const GridMap& grid)          minplus_oracle.hpp:380
 * Grows the index: S -> S*g, H -> H+1.  Existing leaves and nodes keep
 * their matrices; leaves and nodes of the new area, and the new root, are
 * built from `observed` (rows x cols; rows = cols = 0 stands for the
 * reference's default empty GridMap, where nothing is passable).          */
htrip_status htrip_lift_root(htrip_index* h, const uint8_t* observed, int32_t rows, int32_t cols);

/* void queryAllPairs(vps, grid, out, HTripQueryScratch&) const
 *                                              minplus_oracle.hpp:337-341
 * out: k*k uint16 row-major.  Diagonal 0 for Free viewpoints, INF rows and
 * columns for viewpoints that are not Free in `observed`.                 */
htrip_status htrip_query_all_pairs(htrip_index* h, const int32_t* vps, int32_t k,
                                   const uint8_t* observed, int32_t rows, int32_t cols,
                                   uint16_t* out);

/* dist_t queryDistance(Point s, Point t, const GridMap&) const
 *                                              minplus_oracle.hpp:312
 * INF unless both cells are Free and inside the index, 0 for s == t, else
 * the exact distance (one query of the two cells).                        */
htrip_status htrip_query_distance(htrip_index* h, int32_t r1, int32_t c1, int32_t r2, int32_t c2,
                                  const uint8_t* observed, int32_t rows, int32_t cols, uint16_t* out);

/* void queryAllPairsIncremental(vps, grid, out, scratch, state) const
 *                                              minplus_oracle.hpp:290-294
 * `state` caches the last matrix with the index's build / root-growth epoch
 * and its count of opening calls, and keeps a query arena of its own with
 * the last launch's port vectors, projections and pair matrix.
 *  - Same viewpoints, same epoch and no opening since: the cached matrix,
 *    without device work (the reference's fast path).
 *  - Same viewpoints (and passability) and only openings since: the
 *    viewpoints whose leaf-to-root chain holds a matrix those openings
 *    listed are re-lifted and only their pairs recomputed (the reference's
 *    version-stamped re-lift, minplus_oracle.cpp:1444-2002); none: cached.
 *  - Otherwise one full query launch.
 * Every case gives the full query's matrix.  *recomputed (optional): 0
 * cached, 1 full query, 2 re-lift of the changed viewpoints.             */
typedef struct htrip_incremental htrip_incremental; /* opaque */
htrip_status htrip_incremental_create(htrip_incremental** out);
htrip_status htrip_incremental_destroy(htrip_incremental* s);
htrip_status htrip_query_all_pairs_incremental(htrip_index* h, htrip_incremental* s, const int32_t* vps, int32_t k,
                                               const uint8_t* observed, int32_t rows, int32_t cols, uint16_t* out,
                                               int32_t* recomputed);

/* Same query with the per-viewpoint passability already decided by the
 * caller (passable[i] != 0 iff viewpoint i is Free).  vps/passable/out are
 * DEVICE pointers; the call is stream-ordered on the index's stream and
 * returns without synchronising (htrip_sync waits).  For k <= 4096 the plan
 * is built on the device (no copy back to the host, no host wait); larger
 * requests are planned on the host.  HTRIP_QUERY_PLANNER=host|device in the
 * environment overrides where queries are planned.                         */
htrip_status htrip_query_all_pairs_dev(htrip_index* h, const int32_t* vps_dev,
                                       const uint8_t* passable_dev, int32_t k,
                                       uint16_t* out_dev);

/* Allocation-free queryAllPairs (no counterpart in the reference).
 * For callers that may not allocate device memory after start-up, e.g. a
 * serving process whose pool allocator already holds all of HBM, or a
 * real-time planning loop where cudaMalloc / cudaFree (which waits for the
 * whole device) are forbidden.  Same arguments, result and errors as
 * htrip_query_all_pairs (host viewpoints and grid in, host k*k matrix out);
 * all device scratch comes from one fixed 64 MiB array compiled into the
 * library, which every GPU that loads it holds until the process exits.
 *  - No cudaMalloc / cudaFree / allocating library routine is called.
 *  - A query whose scratch would exceed 64 MiB is rejected with
 *    HTRIP_ERR_UNSUPPORTED and a message giving the bytes it needs (it
 *    grows with k^2 and with k times the map side).
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress); make that first call before any stream capture.
 *  - All calls on a device share the array and it keeps the last call's
 *    contents (every call clears what must start cleared).  Calls that
 *    overlapped on the GPU would race on it, so this entry point holds a
 *    process-wide lock until its result is on the host.                   */
htrip_status htrip_query_all_pairs_noalloc(htrip_index* h, const int32_t* vps, int32_t k,
                                           const uint8_t* observed, int32_t rows, int32_t cols,
                                           uint16_t* out);

/* Batched calls over many indexes (maps) of one device.
 *
 * The reference serves one map per call; a host that keeps many maps (one
 * per robot team or session, robot_simulator.cpp:897-1045 keeps two oracles
 * per map) calls MinPlusOracle::queryAllPairs / onBatchCellsOpened once per
 * map.  A batch handle owns a CUDA stream and a scratch arena; one
 * htrip_query_batch call answers every request in ONE launch of the
 * persistent query kernel, and each result is bit-identical to the
 * htrip_query_all_pairs call of the same request alone.                   */
typedef struct htrip_batch htrip_batch; /* opaque */

typedef struct {
    htrip_index* index;       /* built index on the batch's device        */
    const int32_t* vps;       /* k (r, c) pairs, host                     */
    int32_t k;
    const uint8_t* observed;  /* rows*cols CellState bytes, host          */
    int32_t rows, cols;
    uint16_t* out;            /* k*k host output                          */
} htrip_query_request;

htrip_status htrip_batch_create(int device, htrip_batch** out);
/* The same with the batch's stream at the device's highest stream priority
 * (high_priority != 0): its kernels' CTAs are scheduled before those of
 * default-priority streams (e.g. queries ahead of concurrent openings).    */
htrip_status htrip_batch_create_priority(int device, int32_t high_priority, htrip_batch** out);
htrip_status htrip_batch_destroy(htrip_batch* b);

/* queryAllPairs of every request (minplus_oracle.hpp:337-341 per request).
 * Several requests may name the same index.  Synchronous on return.       */
htrip_status htrip_query_batch(htrip_batch* b, const htrip_query_request* reqs, int32_t n);

typedef struct {
    htrip_index* index;       /* built index on the batch's device        */
    const int32_t* rc;        /* n (r, c) cells, host, already set Free   */
    int32_t n;
    const uint8_t* observed;  /* rows*cols CellState bytes, host          */
    int32_t rows, cols;
} htrip_open_request;

/* onBatchCellsOpened of every request (minplus_oracle.hpp:171 per request).
 * The openings of all indexes advance level by level together (each index
 * on its own stream, one host wait per stage for all of them); requests on
 * the same index are applied in call order.  Each index ends in the state,
 * and with the last_batch_stats, of the same calls made one by one.       */
htrip_status htrip_open_batch(htrip_batch* b, const htrip_open_request* reqs, int32_t n);

/* Device time of the batch's last query launch.                           */
htrip_status htrip_batch_last_kernel_ms(const htrip_batch* b, float* ms);

/* Request server over many resident map sessions (no reference
 * counterpart; it generalises the reference simulator's double-buffered
 * update / query threads, robot_simulator.cpp:897-1045, to many maps).
 *  - A session is one map: the server builds its index (MinPlusOracle::
 *    build) and keeps its own copy of the observed grid.
 *  - Requests are asynchronous: a query (queryAllPairs, result written to
 *    the caller's k*k buffer) or an opening (onBatchCellsOpened; the server
 *    marks the cells Free in its grid first).  Requests of one session run
 *    in submission order; requests of different sessions are batched: all
 *    ready queries go into one launch of the query kernel and all ready
 *    openings advance together, while new requests queue for the next
 *    launch (continuous batching).  Every result equals the same request
 *    run alone on a session that saw the same earlier requests.
 *  - Sessions are admitted against an HBM budget by their estimated
 *    footprint; idle sessions are offloaded to host memory (least recently
 *    used first) to make room, and brought back when a request needs them.
 *    A session that cannot fit is refused with HTRIP_ERR_OOM.
 *  - Latency = submission to result in host memory.                       */
typedef struct htrip_server htrip_server; /* opaque */

typedef struct {
    int32_t device;
    uint64_t hbm_budget_bytes;        /* 0: 80% of the device's free memory   */
    int32_t max_requests_per_launch;  /* 0: 128                               */
    int32_t plain_per_call;           /* 1: no batching - one worker serves one
                                         request at a time in arrival order
                                         through the single-index calls (the
                                         baseline the batched server is
                                         measured against)                     */
    int32_t double_buffer;            /* 1: every session keeps two indexes, as
                                         the reference simulator's update thread
                                         does (robot_simulator.cpp:987-1037):
                                         queries read the published one and
                                         never wait behind the session's
                                         openings, which update the other one
                                         and then publish it (twice the memory;
                                         a query may not include openings still
                                         being applied - htrip_server_wait_version
                                         says which it includes)               */
} htrip_server_config;

typedef struct {
    uint64_t launches_query, launches_open;   /* batched launches issued       */
    uint64_t requests_query, requests_open;   /* requests submitted            */
    uint64_t evictions, restores;             /* offloads to / returns from host */
    uint64_t sessions, resident_sessions;
    uint64_t resident_bytes, budget_bytes;
    uint64_t busy_query_us, busy_open_us;     /* time the workers spent in their calls */
} htrip_server_stats;

typedef struct {
    int64_t session;
    int32_t kind;       /* 0 = query (rc = viewpoints, out = k*k), 1 = opening */
    const int32_t* rc;  /* n (r, c) pairs, host                                */
    int32_t n;
    uint16_t* out;
} htrip_server_request;

/* Last error message of a server call on the calling thread.              */
const char* htrip_server_last_error(void);
htrip_status htrip_server_create(const htrip_server_config* cfg, htrip_server** out);
/* Waits for every queued request, then frees all sessions.                */
htrip_status htrip_server_destroy(htrip_server* s);
htrip_status htrip_server_add_session(htrip_server* s, htrip_config cfg, const uint8_t* observed, int32_t rows,
                                      int32_t cols, int64_t* session);
/* Waits for the session's queued requests, then frees it.                 */
htrip_status htrip_server_remove_session(htrip_server* s, int64_t session);
htrip_status htrip_server_submit_query(htrip_server* s, int64_t session, const int32_t* vps, int32_t k,
                                       uint16_t* out, uint64_t* ticket);
htrip_status htrip_server_submit_open(htrip_server* s, int64_t session, const int32_t* rc, int32_t n,
                                      uint64_t* ticket);
/* Blocks until the request is done; returns its status and latency.      */
htrip_status htrip_server_wait(htrip_server* s, uint64_t ticket, double* latency_ms);
/* Same, and *version: for a query, the number of the session's openings
 * (in submission order) its result includes - all earlier ones, unless the
 * server is double-buffered; for an opening, its own number.              */
htrip_status htrip_server_wait_version(htrip_server* s, uint64_t ticket, double* latency_ms, uint64_t* version);
htrip_status htrip_server_get_stats(htrip_server* s, htrip_server_stats* out);
/* Open-loop load: request i is submitted arrival_s[i] seconds after the
 * call starts, by the calling thread; then every request is waited for.
 * latency_ms[i] = its latency (-1 if it failed); wall_s = whole call.     */
htrip_status htrip_server_run_trace(htrip_server* s, const htrip_server_request* reqs, const double* arrival_s,
                                    int32_t n, double* latency_ms, double* wall_s);

/* Measurement helpers (no reference counterpart).
 * htrip_query_work: the algorithmic HBM bytes and min-plus operations of a
 * queryAllPairs on these viewpoints: k*(4b-4) level-0 gathers; per level and
 * node, per child holding viewpoints a lift of nP*nExt entries (below the
 * root), per child pair a meet block of nP*nP, per child with >= 2
 * viewpoints an intra-child block of nP*nP (2 bytes each); operations
 * |V|*nP*nExt per lift, |V1|*nP*nP + |V1|*|V2|*nP per meet, |V|*nP*nP +
 * |V|^2*nP per intra-child block.
 * htrip_last_query_kernel_ms: device time of the last query kernel.
 * htrip_last_query_io: host<->device bytes the last query call copied.     */
htrip_status htrip_query_work(const htrip_index* h, const int32_t* vps, int32_t k, const uint8_t* observed,
                              int32_t rows, int32_t cols, uint64_t* alg_bytes, uint64_t* alg_ops);
htrip_status htrip_last_query_kernel_ms(const htrip_index* h, float* ms);

/* Executed work of the query kernel (no reference counterpart; a
 * measurement mode, off by default).  While counting is on, every query
 * launch of the index that serves it alone counts, per operand row the
 * kernel streamed, the tile entries it updated (rows x tile rows x tile
 * columns), and the rows it skipped because the tile held no finite value:
 * the work actually done, beside htrip_query_work's dense count.
 * htrip_last_query_executed reads the counters of the last launch.       */
htrip_status htrip_set_query_work_counting(htrip_index* h, int32_t on);
htrip_status htrip_last_query_executed(htrip_index* h, uint64_t* entries, uint64_t* rows, uint64_t* skipped);
htrip_status htrip_last_query_io(const htrip_index* h, uint64_t* h2d_bytes, uint64_t* d2h_bytes);

/* Register-only rate (entries/s) of the packed-u16 clamped min-plus update
 * on every SM of `device`: the integer-issue peak the kernels are measured
 * against.  variant 0: add.u16x2 / min.u16x2 clamped form (any a <= INF);
 * 1: the same with the fused add+min intrinsic; 2, 3: the unclamped forms
 * (a <= 5535); 4: min with a saturating packed add (any a <= INF).        */
htrip_status htrip_measure_minplus_rate(int device, int variant, double* entries_per_s);

/* Query tile autotuner (no reference counterpart).  The query kernel has
 * hb::kNumQueryConfigs tile shapes; a process-wide table maps a request
 * bucket (H, root matrix order, log2 of the viewpoint count, log2 of the
 * largest root child group) to the shape to use, falling back to a fixed
 * rule.  htrip_autotune_query times every shape on this request (reps
 * timed launches each, minimum kept), stores the fastest for its bucket and
 * returns it.  Results do not depend on the shape (the kernel is exact for
 * all of them).  The table is exported / imported as text lines
 * "H NP log2_k log2_group cfg"; htrip_autotune_clear empties it.           */
htrip_status htrip_autotune_query(htrip_index* h, const int32_t* vps, int32_t k, const uint8_t* observed,
                                  int32_t rows, int32_t cols, int32_t reps, int32_t* best_cfg, float* best_ms);
htrip_status htrip_autotune_export(char* buf, size_t cap, size_t* len);
htrip_status htrip_autotune_import(const char* text);
htrip_status htrip_autotune_clear(void);

/* Algorithmic work of the index's last opening call (htrip_open_cells,
 * htrip_open_cell or its part of htrip_open_batch): per dirty matrix of
 * order n (b^2 or nV) closed over the pivot set K, n^2 |K| min-plus
 * operations and 2 n^2 2 + |K| n 2 2 bytes, summed over leaves and nodes.  */
htrip_status htrip_last_open_work(const htrip_index* h, uint64_t* alg_bytes, uint64_t* alg_ops);

/* Phase durations of the index's last device-driven opening launch (no
 * reference counterpart): ns[i] = global-timer nanoseconds of phase i of the
 * persistent opening kernel, in order: the seam-node stamping, then per level
 * with work either one phase (matrices of padded order <= 128, updated
 * whole in shared memory) or the insert and compact phases and one phase per
 * closure round (panel and update).  *n = phases recorded.               */
htrip_status htrip_last_open_trace(htrip_index* h, uint64_t* ns, int32_t max_n, int32_t* n);

/* Per level l = 0..H of the index's last opening call (no reference
 * counterpart): out[4l] matrices updated, out[4l+1] the sum of their pivot
 * counts, out[4l+2] the largest pivot count, out[4l+3] closure rounds of
 * 64 pivots.  Writes min(max_levels, H + 1) levels; *n_levels = H + 1.     */
htrip_status htrip_last_open_levels(const htrip_index* h, int64_t* out, int32_t max_levels, int32_t* n_levels);

/* Phase trace of the last query launch of an index / a batch: ns[i] =
 * global-timer nanoseconds of phase i of the persistent query kernel
 * (0: level-0 gathers; 1..H+1: projections of level i with the meets of
 * level i-1; H+2: output).  Barrier schedule (HTRIP_QUERY_DATAFLOW=0): the
 * phase as its first CTA sees it; with max_n >= 2 * phases, ns[phases + i]
 * is the part of phase i until its last CTA finished its work (the rest is
 * the grid-barrier wait).  Dataflow schedule (default; phases overlap): the
 * time from the end of the last unit of phase i-1 (the launch start for
 * i = 0) to the end of the last unit of phase i, in both halves.  *n =
 * entries written.                                                        */
htrip_status htrip_last_query_phases(const htrip_index* h, uint64_t* ns, int32_t max_n, int32_t* n);
htrip_status htrip_batch_last_phases(const htrip_batch* b, uint64_t* ns, int32_t max_n, int32_t* n);

/* Failure-detection self-test (no reference counterpart).  Every wait in
 * the query kernel's grid barrier (barrier schedule, HTRIP_QUERY_DATAFLOW=0)
 * is bounded: after a poll limit the CTA
 * records a timeout in the launch's status word and returns, and the host
 * call fails with HTRIP_ERR_CUDA while the context stays usable.  This runs
 * a 4-CTA launch of the same barrier that can never complete (it expects a
 * fifth CTA) with a short limit: *status = 1 (timeout recorded),
 * *ctas_returned = 4, *ms = the launch's duration.                        */
htrip_status htrip_selftest_barrier_timeout(int device, int32_t* status, int32_t* ctas_returned, float* ms);

/* The same for the completion-counter waits of the query kernel's default
 * (dataflow) schedule: a 4-CTA launch in which every CTA waits for a count
 * that nothing adds, with a short poll limit: *status = 1, *ctas_returned =
 * 4, *ms = the launch's duration.                                          */
htrip_status htrip_selftest_wait_timeout(int device, int32_t* status, int32_t* ctas_returned, float* ms);

/* Wait for all work queued on the index's stream.                         */
htrip_status htrip_sync(htrip_index* h);

/* The index's CUDA stream (a cudaStream_t) for callers that order their own
 * work after stream-ordered calls.                                        */
void* htrip_stream(htrip_index* h);

/* public members S, H, num_leaf_tiles_x (minplus_oracle.hpp:42-45)        */
htrip_status htrip_shape(const htrip_index* h, int32_t* S, int32_t* H, int32_t* leaves_x);

/* last_batch_stats                             minplus_oracle.hpp:256     */
htrip_status htrip_last_batch_stats(const htrip_index* h, htrip_batch_stats* out);

/* size_t totalMemoryBytes() const              minplus_oracle.hpp:385
 * reference_bytes: the reference's accounting of the same index (D, S,
 * D_U, S_U and child_to_ext sizes, minplus_oracle.cpp:2116-2134);
 * device_bytes: HBM actually held by this index.                         */
htrip_status htrip_memory_bytes(const htrip_index* h, uint64_t* reference_bytes,
                                uint64_t* device_bytes);

/* State read-back for bitwise comparison with the reference's public
 * members (host output arrays):
 *   leaves[i].D   (b^2 x b^2)          leaf_tile.hpp:70
 *   leaves[i].S   ((4b-4)^2)           leaf_tile.hpp:71
 *   levels[l-1][n].D_U (nV x nV)       internal_node.hpp:53
 *   levels[l-1][n].S_U (nExt x nExt)   internal_node.hpp:54
 *   levels[l-1][n].child_to_ext[q] (nP x nExt)  internal_node.hpp:55
 * `n` is the row-major node index at level l (tileIndexAtLevel).          */
htrip_status htrip_read_leaf_D(const htrip_index* h, int32_t leaf, uint16_t* out);
htrip_status htrip_read_leaf_S(const htrip_index* h, int32_t leaf, uint16_t* out);
htrip_status htrip_read_node_DU(const htrip_index* h, int32_t lvl, int32_t node, uint16_t* out);
htrip_status htrip_read_node_SU(const htrip_index* h, int32_t lvl, int32_t node, uint16_t* out);
htrip_status htrip_read_node_C2E(const htrip_index* h, int32_t lvl, int32_t node, int32_t quad,
                                 uint16_t* out);
/* Residency (no reference counterpart; the reference keeps every oracle in
 * host RAM).  htrip_offload copies the index's matrices to host memory and
 * frees all of its device memory; every call except htrip_restore,
 * htrip_destroy, htrip_shape, htrip_memory_bytes and htrip_is_resident then
 * fails with HTRIP_ERR_INVALID.  htrip_restore brings it back unchanged
 * (on HTRIP_ERR_OOM it stays offloaded).  htrip_estimate_bytes: the device
 * bytes an index of this config and grid holds after build (matrices,
 * pivot lists and tables; query and update scratch excluded).            */
htrip_status htrip_offload(htrip_index* h);
htrip_status htrip_restore(htrip_index* h);
htrip_status htrip_is_resident(const htrip_index* h, int32_t* resident);
htrip_status htrip_estimate_bytes(htrip_config cfg, int32_t rows, int32_t cols, uint64_t* device_bytes);

/* Canonical per-level checksum of the whole index (no reference
 * counterpart; computed on the device, nothing large is copied):
 *   out[l] = sum mod 2^64 over the level's matrices m (leaves[m].D for
 *   l = 0, levels[l-1][m].D_U above) and logical entries (i, j) of
 *   splitmix64(((m*n + i)*n + j) << 16 | value),  n = b^2 or nV.
 * Two indexes with equal digests hold equal matrices (up to 64-bit hash
 * collisions); the reference's members give the same numbers when summed
 * the same way.  n_out >= H + 1.                                          */
htrip_status htrip_state_digest(const htrip_index* h, uint64_t* out, int32_t n_out);

/* nV, nExt and per-child port count nP of level `lvl` (0 = leaves: n=b^2). */
htrip_status htrip_level_dims(const htrip_index* h, int32_t lvl, int32_t* n, int32_t* n_ext,
                              int32_t* n_child_ports, int32_t* n_nodes);

#ifdef __cplusplus
}
#endif
#endif /* HTRIP_B200_H */
