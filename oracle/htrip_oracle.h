/* Plain-C restatement of the reference's min-plus hierarchy (ozaslan/htrip).
 *
 * TEST INFRASTRUCTURE ONLY: this is the CPU checker used by tests/ (and
 * pinned against the reference's own known-answer vectors and against the
 * compiled reference in oracle/_ref).  The product never links it.
 *
 * Grids are uint8 CellState arrays (0 Unknown, 1 Free, 2 Obstacle), cells
 * are int32 (r, c) pairs, distances uint16 with INF = 60000.
 */
#ifndef HTRIP_ORACLE_H
#define HTRIP_ORACLE_H
#include <stdint.h>

typedef struct orc orc_t;

orc_t* orc_create(int b, int g);
void orc_destroy(orc_t* o);
/* 1 on success, 0 where MinPlusOracle::build returns false. */
int orc_build(orc_t* o, const uint8_t* observed, int rows, int cols);
void orc_open_batch(orc_t* o, const int32_t* rc, int n, const uint8_t* observed, int rows, int cols);
void orc_query(const orc_t* o, const int32_t* vps, int k, const uint8_t* observed, int rows, int cols,
               uint16_t* out);
void orc_stats(const orc_t* o, int32_t* out3);
int orc_S(const orc_t* o);
int orc_H(const orc_t* o);
/* Copies of the state matrices; each returns the matrix order. */
int orc_leaf_D(const orc_t* o, int leaf, uint16_t* out);
int orc_node_DU(const orc_t* o, int lvl, int node, uint16_t* out);
/* k one-to-all BFS runs (reference BfsOracle::queryAllPairs). */
void orc_bfs_all_pairs(const uint8_t* observed, int rows, int cols, const int32_t* vps, int k, uint16_t* out);

#endif
