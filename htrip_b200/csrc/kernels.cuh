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
void launch_leaf_bfs(const uint8_t* pass, int S, int b, int leaves_x, int n_leaves, MatSet leaves,
                     cudaStream_t st);

// Internal-node initial D_U: block diagonal of child summaries, INF
// elsewhere (internal_node.cpp:98-145).  child_ext: the child level's
// port -> matrix-index table (nP entries).
void launch_node_init(MatSet node, MatSet child, const int* child_ext, int nP, int g, int nodes_x,
                      int child_nodes_x, int n_nodes, cudaStream_t st);

// Seam edges of the build (internal_node.cpp:155-173): seams = 6 ints per
// candidate {u, v, ur, uc, vr, vc} (node-relative coordinates).
void launch_seams_build(MatSet node, const int* seams, int n_seams, const uint8_t* pass, int S,
                        int side, int nodes_x, int n_nodes, uint8_t* kflag, cudaStream_t st);

// --- closure over pivot sets -------------------------------------------------
// Compact per-matrix pivot flags into sorted lists (clears the flags).
void launch_compact_pivots(uint8_t* kflag, int NP, const int* active, int n_active, int* klist,
                           int* kcnt, cudaStream_t st);

// One round of the blocked pivot-set Kleene closure: pivots
// klist[m][round*B .. round*B+B).  panel/flags: scratch for n_active mats.
void launch_closure_round(MatSet M, const int* active, int n_active, const int* klist,
                          const int* kcnt, int round, uint16_t* panel, uint8_t* flags,
                          cudaStream_t st);

// --- incremental updates -----------------------------------------------------
// Insert opened in-leaf edges (leaf_tile.cpp:311-330).  edges: per active
// leaf a range [eoff[i], eoff[i+1]) of (u, v) pairs (2 ints).  Marks pivot
// flags, counts pivots into *pivots.
void launch_leaf_edges(MatSet leaves, const int* active, int n_active, const int* eoff,
                       const int* edges, uint8_t* kflag, int* pivots, cudaStream_t st);

// Child-summary decreases into parent D_U (internal_node.cpp:343-353):
// for each active node and each child whose flag is set, insert every
// child summary entry smaller than the parent's and mark both endpoints.
void launch_node_child_insert(MatSet node, MatSet child, const int* child_ext, int nP, int g,
                              int nodes_x, int child_nodes_x, const int* active, int n_active,
                              const uint8_t* child_dec, uint8_t* kflag, cudaStream_t st);

// Seam edges of an update (internal_node.cpp:356-365): per active node a
// range [soff[i], soff[i+1]) of (u, v) V_U-index pairs.
void launch_node_seams(MatSet node, const int* active, int n_active, const int* soff,
                       const int* seams, uint8_t* kflag, cudaStream_t st);

// Snapshot / compare of a matrix's exterior block (summary S or S_U):
// snap[i] holds nExt*nExt entries per active matrix.  compare sets
// dec[active[i]] = 1 when any entry decreased (refreshBoundarySummary,
// leaf_tile.cpp:253-273, internal_node.cpp:415-433).
void launch_ext_snapshot(MatSet M, const int* ext, int nExt, const int* active, int n_active,
                         uint16_t* snap, cudaStream_t st);
void launch_ext_compare(MatSet M, const int* ext, int nExt, const int* active, int n_active,
                        const uint16_t* snap, uint8_t* dec, cudaStream_t st);

// --- query -------------------------------------------------------------------
// Level-0 extraction (minplus_oracle.cpp:990-1048): X0t[p*ldx + j] =
// leaf D[u_j][ext[p]] for viewpoint j (sorted order), and same-leaf pairs
// into M (k x k, sorted order).  vp: per sorted viewpoint {leaf, u, leaf
// group start, leaf group end} (4 ints).
void launch_query_level0(MatSet leaves, const int* ext, int nExt, const int* vp, int k, uint16_t* X0t,
                         int ldx, uint16_t* M, int ldm, cudaStream_t st);

// Grouped gather-GEMM Y[i][:] = min_p X[i][p] + D_U[off + p][:] for the
// viewpoints i of each child group.  groups: 4 ints {node, quad, start,
// count} per group.  Active port lists are built inside.
void launch_query_project(MatSet node, int nP, const int* groups, int n_groups, int max_group,
                          const uint16_t* Xt, int ldx, uint16_t* Y, int ldy, int* kidx,
                          cudaStream_t st);

// Lift X_next t[e][j] = Y[j][ext[e]] for all viewpoints j in [0, k).
void launch_query_lift(const uint16_t* Y, int ldy, const int* ext, int nExt, int k, uint16_t* Xt_next,
                       int ldx, cudaStream_t st);

// Meet: for every node group (range [start, end) of sorted viewpoints) and
// i < j in it: M[i][j] = min(M[i][j], min_p Y[i][qoff[j]+p] + Xt[p][j]).
// ngroups: 3 ints {start, end, first child group} per node; qoff[j] = the
// V_U offset of viewpoint j's child block.
void launch_query_meet(const int* ngroups, int n_ngroups, const int* qoff, const uint16_t* Y, int ldy,
                       const uint16_t* Xt, int ldx, int nP, uint16_t* M, int ldm, int max_w,
                       cudaStream_t st);

// Final un-permute: out[a*k + c] = M[inv[a]][inv[c]]; rows/cols of
// non-passable viewpoints INF, diagonal 0 for passable ones.
void launch_query_finalize(const uint16_t* M, int ldm, const int* inv, int k, uint16_t* out,
                           cudaStream_t st);

// ptr[0 .. n) = value.
void launch_fill_u16(uint16_t* ptr, size_t n, uint16_t value, cudaStream_t st);

// Gather an exterior block (S / S_U / child_to_ext) of one matrix to dense.
void launch_gather_block(const uint16_t* mat, int NP, const int* rows, int nr, const int* cols, int nc,
                         uint16_t* out, cudaStream_t st);

}  // namespace hb
