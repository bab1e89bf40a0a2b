/* Plain-C restatement of the reference HTRIP min-plus hierarchy.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU checker).  Each function names the
 * reference code it restates (paths inside ozaslan/htrip).  Arithmetic is
 * the reference's: dist_t = uint16, INF = 60000, add_dist(a, b) =
 * min(a + b, INF) (include/htrip/types.hpp:34,45,66-70).
 */
#include "htrip_oracle.h"

#include <stdlib.h>
#include <string.h>

#define INF 60000u

/* add_dist, types.hpp:66-70 */
static uint16_t add_d(uint32_t a, uint32_t b) {
    if (a >= INF || b >= INF) return (uint16_t)INF;
    uint32_t s = a + b;
    return (uint16_t)(s >= INF ? INF : s);
}

typedef struct {
    int *p; int n, cap;
} ivec;
static void iv_push(ivec* v, int x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 16;
        v->p = (int*)realloc(v->p, (size_t)v->cap * sizeof(int));
    }
    v->p[v->n++] = x;
}

typedef struct {
    int side, cs, n, nP, nExt, nodes_x, nnodes;
    int* ext;    /* exterior port e -> matrix index (leaf cell / V_U index) */
    int nseams;
    int* seam;   /* 6 ints per seam candidate: u, v, ur, uc, vr, vc (node-local) */
    uint16_t* mat;
} lev_t;

struct orc {
    int b, g, S, H, leaves_x, built;
    lev_t* L;
    int32_t stats[3];
};

/* getTilePorts, leaf_tile.cpp:11-30 */
static void port_local(int s, int p, int* r, int* c) {
    if (p < s) { *r = 0; *c = p; }
    else if (p < 2 * s) { *r = s - 1; *c = p - s; }
    else if (p < 3 * s - 2) { *r = p - 2 * s + 1; *c = 0; }
    else { *r = p - (3 * s - 2) + 1; *c = s - 1; }
}

/* getPortIndexInTile, internal_node.cpp:290-304 */
static int port_index(int r, int c, int s) {
    if (r == 0 && c >= 0 && c < s) return c;
    if (r == s - 1 && c >= 0 && c < s) return s + c;
    if (c == 0 && r > 0 && r < s - 1) return 2 * s + r - 1;
    if (c == s - 1 && r > 0 && r < s - 1) return 3 * s - 2 + r - 1;
    return -1;
}

/* V_U index of node-local (r, c): InternalNode ctor V_U / findVertexIndex
 * (internal_node.cpp:29-42, :306-319). */
static int vidx(const lev_t* L, int g, int r, int c) {
    if (r < 0 || c < 0 || r >= L->side || c >= L->side) return -1;
    int q = (r / L->cs) * g + (c / L->cs);
    int p = port_index(r % L->cs, c % L->cs, L->cs);
    return p < 0 ? -1 : q * L->nP + p;
}

static uint16_t* M_(const lev_t* L, int m) { return L->mat + (size_t)m * L->n * L->n; }

static int passable(const uint8_t* obs, int rows, int cols, int r, int c) {
    return r >= 0 && c >= 0 && r < rows && c < cols && obs[(size_t)r * cols + c] == 1;
}

orc_t* orc_create(int b, int g) {
    orc_t* o = (orc_t*)calloc(1, sizeof(orc_t));
    o->b = b;
    o->g = g;
    return o;
}

static void free_levels(orc_t* o) {
    if (!o->L) return;
    for (int l = 0; l <= o->H; ++l) {
        free(o->L[l].ext);
        free(o->L[l].seam);
        free(o->L[l].mat);
    }
    free(o->L);
    o->L = NULL;
}

void orc_destroy(orc_t* o) {
    if (!o) return;
    free_levels(o);
    free(o);
}

static void identity(uint16_t* D, int n) {
    for (size_t i = 0; i < (size_t)n * n; ++i) D[i] = (uint16_t)INF;
    for (int i = 0; i < n; ++i) D[(size_t)i * n + i] = 0;
}

/* Sequential relaxation over pivots K (leaf_tile.cpp:348-371,
 * internal_node.cpp:201-231, :372-399): for each k, every row i with a
 * finite D[k][i] takes min(row_i, D[k][i] + row_k). */
static void relax_pivots(uint16_t* D, int n, const int* K, int nk) {
    for (int t = 0; t < nk; ++t) {
        const int k = K[t];
        const uint16_t* rk = D + (size_t)k * n;
        for (int i = 0; i < n; ++i) {
            const uint16_t dik = rk[i];
            if (dik >= INF) continue;
            uint16_t* ri = D + (size_t)i * n;
            for (int j = 0; j < n; ++j) {
                const uint16_t alt = add_d(dik, rk[j]);
                if (alt < ri[j]) ri[j] = alt;
            }
        }
    }
}

/* LeafTile::recomputeFromGrid, leaf_tile.cpp:56-153 (unit weights). */
static void leaf_build(orc_t* o, int leaf, const uint8_t* obs, int rows, int cols, int* q) {
    const int b = o->b, n = b * b;
    const int ty = leaf / o->leaves_x, tx = leaf % o->leaves_x;
    const int R0 = ty * b, C0 = tx * b;
    uint16_t* D = M_(&o->L[0], leaf);
    identity(D, n);
    for (int i = 0; i < n; ++i) {
        if (!passable(obs, rows, cols, R0 + i / b, C0 + i % b)) continue;
        uint16_t* row = D + (size_t)i * n;
        int head = 0, tail = 0;
        q[tail++] = i;
        while (head < tail) {
            const int u = q[head++];
            const int ur = u / b, uc = u % b;
            const uint16_t alt = (uint16_t)(row[u] + 1);
            const int nb[4][2] = {{ur - 1, uc}, {ur + 1, uc}, {ur, uc - 1}, {ur, uc + 1}};
            for (int d = 0; d < 4; ++d) {
                const int vr = nb[d][0], vc = nb[d][1];
                if (vr < 0 || vc < 0 || vr >= b || vc >= b) continue;
                const int v = vr * b + vc;
                if (passable(obs, rows, cols, R0 + vr, C0 + vc) && row[v] == INF) {
                    row[v] = alt;
                    q[tail++] = v;
                }
            }
        }
    }
}

static int child_index(const orc_t* o, int l, int node, int q) {
    const lev_t* Lv = &o->L[l];
    const lev_t* Lc = &o->L[l - 1];
    const int tx = node % Lv->nodes_x, ty = node / Lv->nodes_x;
    return (ty * o->g + q / o->g) * Lc->nodes_x + (tx * o->g + q % o->g);
}

/* InternalNode::recomputeFromChildren, internal_node.cpp:94-245. */
static void node_build(orc_t* o, int l, int node, const uint8_t* obs, int rows, int cols) {
    lev_t* Lv = &o->L[l];
    const lev_t* Lc = &o->L[l - 1];
    const int n = Lv->n, nP = Lv->nP, g = o->g;
    uint16_t* D = M_(Lv, node);
    identity(D, n);
    for (int q = 0; q < g * g; ++q) {
        const uint16_t* C = M_(Lc, child_index(o, l, node, q));
        for (int a = 0; a < nP; ++a)
            for (int c = 0; c < nP; ++c) {
                const uint16_t w = C[(size_t)Lc->ext[a] * Lc->n + Lc->ext[c]];
                uint16_t* d = &D[(size_t)(q * nP + a) * n + q * nP + c];
                if (w < INF && w < *d) *d = w;
            }
    }
    const int R0 = (node / Lv->nodes_x) * Lv->side, C0 = (node % Lv->nodes_x) * Lv->side;
    char* in = (char*)calloc((size_t)n, 1);
    ivec K = {0};
    for (int s = 0; s < Lv->nseams; ++s) {
        const int* e = Lv->seam + 6 * s;
        if (!passable(obs, rows, cols, R0 + e[2], C0 + e[3]) || !passable(obs, rows, cols, R0 + e[4], C0 + e[5]))
            continue;
        if (1 < D[(size_t)e[0] * n + e[1]]) D[(size_t)e[0] * n + e[1]] = 1;
        if (1 < D[(size_t)e[1] * n + e[0]]) D[(size_t)e[1] * n + e[0]] = 1;
        if (!in[e[0]]) { in[e[0]] = 1; iv_push(&K, e[0]); }
        if (!in[e[1]]) { in[e[1]] = 1; iv_push(&K, e[1]); }
    }
    relax_pivots(D, n, K.p, K.n);
    free(K.p);
    free(in);
}

static void make_levels(orc_t* o) {
    const int b = o->b, g = o->g;
    o->L = (lev_t*)calloc((size_t)o->H + 1, sizeof(lev_t));
    lev_t* L0 = &o->L[0];
    L0->side = b;
    L0->n = b * b;
    L0->nExt = 4 * b - 4;
    L0->nodes_x = o->S / b;
    L0->nnodes = L0->nodes_x * L0->nodes_x;
    L0->ext = (int*)malloc(sizeof(int) * (size_t)L0->nExt);
    for (int e = 0; e < L0->nExt; ++e) {
        int r, c;
        port_local(b, e, &r, &c);
        L0->ext[e] = r * b + c;
    }
    L0->mat = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)L0->nnodes * L0->n * L0->n);
    int cs = b;
    for (int l = 1; l <= o->H; ++l) {
        lev_t* Lv = &o->L[l];
        Lv->cs = cs;
        Lv->side = cs * g;
        Lv->nP = 4 * cs - 4;
        Lv->n = g * g * Lv->nP;
        Lv->nExt = 4 * Lv->side - 4;
        Lv->nodes_x = o->S / Lv->side;
        Lv->nnodes = Lv->nodes_x * Lv->nodes_x;
        Lv->ext = (int*)malloc(sizeof(int) * (size_t)Lv->nExt);
        for (int e = 0; e < Lv->nExt; ++e) {
            int r, c;
            port_local(Lv->side, e, &r, &c);
            Lv->ext[e] = vidx(Lv, g, r, c);
        }
        /* seam candidates: touching port pairs of different children (internal_node.cpp:72-89) */
        ivec sv = {0};
        for (int u = 0; u < Lv->n; ++u) {
            const int q = u / Lv->nP;
            int pr, pc;
            port_local(cs, u % Lv->nP, &pr, &pc);
            const int r = (q / g) * cs + pr, c = (q % g) * cs + pc;
            const int nb[2][2] = {{r, c + 1}, {r + 1, c}};
            for (int d = 0; d < 2; ++d) {
                const int v = vidx(Lv, g, nb[d][0], nb[d][1]);
                if (v < 0 || v / Lv->nP == q) continue;
                iv_push(&sv, u); iv_push(&sv, v); iv_push(&sv, r); iv_push(&sv, c);
                iv_push(&sv, nb[d][0]); iv_push(&sv, nb[d][1]);
            }
        }
        Lv->seam = sv.p;
        Lv->nseams = sv.n / 6;
        Lv->mat = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)Lv->nnodes * Lv->n * Lv->n);
        cs *= g;
    }
}

/* MinPlusOracle::build, minplus_oracle.cpp:48-137 */
int orc_build(orc_t* o, const uint8_t* obs, int rows, int cols) {
    const int b = o->b, g = o->g;
    if (!(b > 0 && g >= 2 && g * g <= 256)) return 0;
    const int mx = rows > cols ? rows : cols;
    if (mx <= 0) return 0;
    free_levels(o);
    int S = b;
    while (S < mx) S *= g;
    int H = 0;
    for (int t = S / b; t > 1; t /= g) ++H;
    o->S = S;
    o->H = H;
    o->leaves_x = S / b;
    make_levels(o);
    int* q = (int*)malloc(sizeof(int) * (size_t)b * b);
    for (int leaf = 0; leaf < o->L[0].nnodes; ++leaf) leaf_build(o, leaf, obs, rows, cols, q);
    free(q);
    for (int l = 1; l <= H; ++l)
        for (int node = 0; node < o->L[l].nnodes; ++node) node_build(o, l, node, obs, rows, cols);
    o->built = 1;
    return 1;
}

typedef struct { int q, a, c; uint16_t w; } cdec_t;  /* ChildDecrease, types.hpp:166-171 */
typedef struct { cdec_t* p; int n, cap; } cdvec;
static void cd_push(cdvec* v, cdec_t x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 16;
        v->p = (cdec_t*)realloc(v->p, (size_t)v->cap * sizeof(cdec_t));
    }
    v->p[v->n++] = x;
}

/* refreshBoundarySummary (leaf_tile.cpp:253-273, internal_node.cpp:415-433):
 * exterior-port pairs whose distance dropped below the snapshot. */
static void ext_decreases(const lev_t* L, const uint16_t* D, const uint16_t* snap, int quad, cdvec* out) {
    for (int a = 0; a < L->nExt; ++a)
        for (int c = 0; c < L->nExt; ++c) {
            const uint16_t w = D[(size_t)L->ext[a] * L->n + L->ext[c]];
            if (w < snap[(size_t)a * L->nExt + c]) {
                cdec_t d = {quad, a, c, w};
                cd_push(out, d);
            }
        }
}

static void ext_snapshot(const lev_t* L, const uint16_t* D, uint16_t* snap) {
    for (int a = 0; a < L->nExt; ++a)
        for (int c = 0; c < L->nExt; ++c) snap[(size_t)a * L->nExt + c] = D[(size_t)L->ext[a] * L->n + L->ext[c]];
}

static int find_lca(const orc_t* o, int r1, int c1, int r2, int c2) { /* minplus_oracle.cpp:24-46 */
    int ax = c1 / o->b, ay = r1 / o->b, bx = c2 / o->b, by = r2 / o->b;
    if (ax == bx && ay == by) return 0;
    for (int l = 1; l <= o->H; ++l) {
        ax /= o->g; ay /= o->g; bx /= o->g; by /= o->g;
        if (ax == bx && ay == by) return l;
    }
    return o->H + 1;
}

/* MinPlusOracle::onBatchCellsOpened, minplus_oracle.cpp:530-729 */
void orc_open_batch(orc_t* o, const int32_t* rc, int n, const uint8_t* obs, int rows, int cols) {
    const int b = o->b, g = o->g, H = o->H, S = o->S;
    lev_t* L0 = &o->L[0];
    o->stats[0] = o->stats[1] = o->stats[2] = 0;
    static const int dr[4] = {-1, 1, 0, 0}, dc[4] = {0, 0, -1, 1};
    /* 1. bucket by leaf (first-touch order) */
    int* slot = (int*)malloc(sizeof(int) * (size_t)L0->nnodes);
    for (int i = 0; i < L0->nnodes; ++i) slot[i] = -1;
    ivec leaves = {0};
    ivec* cells = NULL;
    for (int i = 0; i < n; ++i) {
        const int r = rc[2 * i], c = rc[2 * i + 1];
        if (r < 0 || c < 0 || r >= S || c >= S) continue;
        const int leaf = (r / b) * o->leaves_x + c / b;
        if (slot[leaf] < 0) {
            slot[leaf] = leaves.n;
            iv_push(&leaves, leaf);
            cells = (ivec*)realloc(cells, sizeof(ivec) * (size_t)leaves.n);
            memset(&cells[leaves.n - 1], 0, sizeof(ivec));
        }
        iv_push(&cells[slot[leaf]], i);
    }
    if (leaves.n == 0) { free(slot); free(leaves.p); free(cells); return; }
    /* 2. seams by LCA level and node (minplus_oracle.cpp:563-598) */
    ivec** seams = (ivec**)calloc((size_t)H + 1, sizeof(ivec*));
    for (int l = 1; l <= H; ++l) seams[l] = (ivec*)calloc((size_t)o->L[l].nnodes, sizeof(ivec));
    for (int i = 0; i < n; ++i) {
        const int r = rc[2 * i], c = rc[2 * i + 1];
        if (r < 0 || c < 0 || r >= S || c >= S) continue;
        const int wok = r < rows && c < cols && obs[(size_t)r * cols + c] != 2; /* edgeWeight < INF */
        for (int d = 0; d < 4; ++d) {
            const int nr = r + dr[d], nc = c + dc[d];
            if (!passable(obs, rows, cols, nr, nc) || !wok) continue;
            if (nr / b == r / b && nc / b == c / b) continue;
            const int lca = find_lca(o, r, c, nr, nc);
            if (lca < 1 || lca > H) continue;
            const lev_t* Lv = &o->L[lca];
            const int node = (r / Lv->side) * Lv->nodes_x + c / Lv->side;
            const int u = vidx(Lv, g, r % Lv->side, c % Lv->side), v = vidx(Lv, g, nr % Lv->side, nc % Lv->side);
            iv_push(&seams[lca][node], u);
            iv_push(&seams[lca][node], v);
        }
    }
    /* 3. leaves (LeafTile::onBatchCellsOpened, leaf_tile.cpp:297-374) */
    cdvec* cur = NULL;
    ivec cur_active = {0};
    if (H > 0) cur = (cdvec*)calloc((size_t)o->L[1].nnodes, sizeof(cdvec));
    int pivots = 0;
    uint16_t* snap = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)L0->nExt * L0->nExt);
    char* in = (char*)calloc((size_t)L0->n, 1);
    for (int li = 0; li < leaves.n; ++li) {
        const int leaf = leaves.p[li];
        const int ty = leaf / o->leaves_x, tx = leaf % o->leaves_x;
        uint16_t* D = M_(L0, leaf);
        ext_snapshot(L0, D, snap);
        ivec K = {0};
        memset(in, 0, (size_t)L0->n);
        for (int t = 0; t < cells[li].n; ++t) {
            const int i = cells[li].p[t];
            const int r = rc[2 * i], c = rc[2 * i + 1];
            const int wok = r < rows && c < cols && obs[(size_t)r * cols + c] != 2;
            if (!wok) continue;
            const int u = (r - ty * b) * b + (c - tx * b);
            for (int d = 0; d < 4; ++d) {
                const int vr = r + dr[d], vc = c + dc[d];
                if (vr < ty * b || vr >= ty * b + b || vc < tx * b || vc >= tx * b + b) continue;
                if (!passable(obs, rows, cols, vr, vc)) continue;
                const int v = (vr - ty * b) * b + (vc - tx * b);
                if (1 < D[(size_t)u * L0->n + v]) {
                    D[(size_t)u * L0->n + v] = 1;
                    D[(size_t)v * L0->n + u] = 1;
                    if (!in[u]) { in[u] = 1; iv_push(&K, u); }
                    if (!in[v]) { in[v] = 1; iv_push(&K, v); }
                }
            }
        }
        pivots += K.n;
        relax_pivots(D, L0->n, K.p, K.n);
        free(K.p);
        if (H > 0) {
            cdvec decs = {0};
            ext_decreases(L0, D, snap, (ty % g) * g + (tx % g), &decs);
            if (decs.n) {
                const int p = (ty / g) * o->L[1].nodes_x + tx / g;
                if (cur[p].n == 0) iv_push(&cur_active, p);
                for (int t = 0; t < decs.n; ++t) cd_push(&cur[p], decs.p[t]);
            }
            free(decs.p);
        }
    }
    free(in);
    free(snap);
    o->stats[0] = leaves.n;
    o->stats[2] = pivots;
    /* 4. levels 1..H (minplus_oracle.cpp:650-722) */
    int dirty = 0;
    for (int l = 1; l <= H; ++l) {
        lev_t* Lv = &o->L[l];
        for (int node = 0; node < Lv->nnodes; ++node)
            if (seams[l][node].n && cur[node].n == 0) {
                int present = 0;
                for (int t = 0; t < cur_active.n; ++t) present |= cur_active.p[t] == node;
                if (!present) iv_push(&cur_active, node);
            }
        dirty += cur_active.n;
        cdvec* next = NULL;
        ivec next_active = {0};
        if (l < H) next = (cdvec*)calloc((size_t)o->L[l + 1].nnodes, sizeof(cdvec));
        uint16_t* snapn = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)Lv->nExt * Lv->nExt);
        char* inn = (char*)calloc((size_t)Lv->n, 1);
        for (int t = 0; t < cur_active.n; ++t) {
            const int node = cur_active.p[t];
            uint16_t* D = M_(Lv, node);
            const int nn = Lv->n;
            ext_snapshot(Lv, D, snapn);
            /* applyConwayPerturbations, internal_node.cpp:332-413 */
            ivec K = {0};
            memset(inn, 0, (size_t)nn);
            for (int e = 0; e < cur[node].n; ++e) {
                const cdec_t* dd = &cur[node].p[e];
                const int u = dd->q * Lv->nP + dd->a, v = dd->q * Lv->nP + dd->c;
                if (dd->w < D[(size_t)u * nn + v]) {
                    D[(size_t)u * nn + v] = dd->w;
                    D[(size_t)v * nn + u] = dd->w;
                    if (!inn[u]) { inn[u] = 1; iv_push(&K, u); }
                    if (!inn[v]) { inn[v] = 1; iv_push(&K, v); }
                }
            }
            for (int e = 0; e + 1 < seams[l][node].n; e += 2) {
                const int u = seams[l][node].p[e], v = seams[l][node].p[e + 1];
                if (u < 0 || v < 0) continue;
                if (1 < D[(size_t)u * nn + v]) {
                    D[(size_t)u * nn + v] = 1;
                    D[(size_t)v * nn + u] = 1;
                    if (!inn[u]) { inn[u] = 1; iv_push(&K, u); }
                    if (!inn[v]) { inn[v] = 1; iv_push(&K, v); }
                }
            }
            if (K.n == 0) { free(K.p); continue; }
            relax_pivots(D, nn, K.p, K.n);
            free(K.p);
            if (l < H) {
                const int px = node % Lv->nodes_x, py = node / Lv->nodes_x;
                cdvec decs = {0};
                ext_decreases(Lv, D, snapn, (py % g) * g + (px % g), &decs);
                if (decs.n) {
                    const int gp = (py / g) * o->L[l + 1].nodes_x + px / g;
                    if (next[gp].n == 0) iv_push(&next_active, gp);
                    for (int e = 0; e < decs.n; ++e) cd_push(&next[gp], decs.p[e]);
                }
                free(decs.p);
            }
        }
        free(inn);
        free(snapn);
        for (int node = 0; node < Lv->nnodes; ++node) free(cur[node].p);
        free(cur);
        free(cur_active.p);
        cur = next;
        cur_active = next_active;
    }
    o->stats[1] = dirty;
    for (int l = 1; l <= H; ++l) {
        for (int node = 0; node < o->L[l].nnodes; ++node) free(seams[l][node].p);
        free(seams[l]);
    }
    free(seams);
    for (int li = 0; li < leaves.n; ++li) free(cells[li].p);
    free(cells);
    free(leaves.p);
    free(slot);
    free(cur_active.p);
}

/* MinPlusOracle::queryAllPairs, minplus_oracle.cpp:934-1419, restated
 * without the Manhattan "closed" pruning (which never changes a result):
 * level-0 port vectors from leaf D, same-leaf pairs from D, then per level
 * the lift X_l = X_{l-1} (x) child_to_ext and the meets of every viewpoint
 * pair that shares the node (different children and same child). */
void orc_query(const orc_t* o, const int32_t* vps, int k, const uint8_t* obs, int rows, int cols, uint16_t* out) {
    const int b = o->b, g = o->g, H = o->H;
    for (size_t i = 0; i < (size_t)k * k; ++i) out[i] = (uint16_t)INF;
    if (k == 0) return;
    char* ok = (char*)calloc((size_t)k, 1);
    int maxExt = 0;
    for (int l = 0; l <= H; ++l) if (o->L[l].nExt > maxExt) maxExt = o->L[l].nExt;
    uint16_t* X = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)k * maxExt);
    uint16_t* Xn = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)k * maxExt);
    int* node = (int*)malloc(sizeof(int) * (size_t)k);
    const lev_t* L0 = &o->L[0];
    for (int i = 0; i < k; ++i) {
        const int r = vps[2 * i], c = vps[2 * i + 1];
        ok[i] = passable(obs, rows, cols, r, c) && r < o->S && c < o->S;
        if (!ok[i]) continue;
        out[(size_t)i * k + i] = 0;
        const int leaf = (r / b) * o->leaves_x + c / b, u = (r % b) * b + c % b;
        node[i] = leaf;
        const uint16_t* row = M_(L0, leaf) + (size_t)u * L0->n;
        for (int p = 0; p < L0->nExt; ++p) X[(size_t)i * maxExt + p] = row[L0->ext[p]];
    }
    for (int i = 0; i < k; ++i)
        for (int j = i + 1; j < k; ++j)
            if (ok[i] && ok[j] && node[i] == node[j]) {
                const int u = (vps[2 * i] % b) * b + vps[2 * i + 1] % b;
                const int v = (vps[2 * j] % b) * b + vps[2 * j + 1] % b;
                const uint16_t d = M_(L0, node[i])[(size_t)u * L0->n + v];
                out[(size_t)i * k + j] = out[(size_t)j * k + i] = d;
            }
    uint16_t* proj = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)(o->H ? o->L[H].n : 1));
    for (int l = 1; l <= H; ++l) {
        const lev_t* Lv = &o->L[l];
        const lev_t* Lc = &o->L[l - 1];
        const int nP = Lv->nP, n = Lv->n;
        for (int i = 0; i < k; ++i) {
            if (!ok[i]) continue;
            const int cx = vps[2 * i + 1] / Lc->side, cy = vps[2 * i] / Lc->side;
            const int nd = (cy / g) * Lv->nodes_x + cx / g;
            const int qi = (cy % g) * g + cx % g;
            const uint16_t* D = M_(Lv, nd);
            const uint16_t* xi = X + (size_t)i * maxExt;
            /* projection of viewpoint i through D_U rows of its child block */
            for (int v = 0; v < n; ++v) proj[v] = (uint16_t)INF;
            for (int p = 0; p < nP; ++p) {
                if (xi[p] >= INF) continue;
                const uint16_t* row = D + (size_t)(qi * nP + p) * n;
                for (int v = 0; v < n; ++v) {
                    const uint16_t a = add_d(xi[p], row[v]);
                    if (a < proj[v]) proj[v] = a;
                }
            }
            /* lift (only below the root): X_l[e] = proj[ext[e]] */
            if (l < H)
                for (int e = 0; e < Lv->nExt; ++e) Xn[(size_t)i * maxExt + e] = proj[Lv->ext[e]];
            /* meets with every later viewpoint of the same node */
            for (int j = i + 1; j < k; ++j) {
                if (!ok[j]) continue;
                const int dx = vps[2 * j + 1] / Lc->side, dy = vps[2 * j] / Lc->side;
                if ((dy / g) * Lv->nodes_x + dx / g != nd) continue;
                const int qj = (dy % g) * g + dx % g;
                const uint16_t* xj = X + (size_t)j * maxExt;
                uint16_t best = out[(size_t)i * k + j];
                for (int p = 0; p < nP; ++p) {
                    const uint16_t a = add_d(proj[qj * nP + p], xj[p]);
                    if (a < best) best = a;
                }
                out[(size_t)i * k + j] = out[(size_t)j * k + i] = best;
            }
        }
        uint16_t* t = X; X = Xn; Xn = t;
    }
    free(proj);
    free(node);
    free(X);
    free(Xn);
    free(ok);
}

void orc_stats(const orc_t* o, int32_t* out3) { memcpy(out3, o->stats, sizeof(o->stats)); }
int orc_S(const orc_t* o) { return o->S; }
int orc_H(const orc_t* o) { return o->H; }

int orc_leaf_D(const orc_t* o, int leaf, uint16_t* out) {
    const lev_t* L0 = &o->L[0];
    if (out) memcpy(out, M_(L0, leaf), sizeof(uint16_t) * (size_t)L0->n * L0->n);
    return L0->n;
}

int orc_node_DU(const orc_t* o, int lvl, int node, uint16_t* out) {
    const lev_t* Lv = &o->L[lvl];
    if (out) memcpy(out, M_(Lv, node), sizeof(uint16_t) * (size_t)Lv->n * Lv->n);
    return Lv->n;
}

/* BfsOracle::queryAllPairs / queryOneToAll, bfs_oracle.cpp:79-202 */
void orc_bfs_all_pairs(const uint8_t* obs, int rows, int cols, const int32_t* vps, int k, uint16_t* out) {
    const size_t N = (size_t)rows * cols;
    uint16_t* dist = (uint16_t*)malloc(sizeof(uint16_t) * (N ? N : 1));
    int* q = (int*)malloc(sizeof(int) * (N ? N : 1));
    for (int i = 0; i < k; ++i) {
        for (int j = 0; j < k; ++j) out[(size_t)i * k + j] = (uint16_t)INF;
        const int sr = vps[2 * i], sc = vps[2 * i + 1];
        if (!passable(obs, rows, cols, sr, sc)) continue;
        for (size_t t = 0; t < N; ++t) dist[t] = (uint16_t)INF;
        int head = 0, tail = 0;
        dist[(size_t)sr * cols + sc] = 0;
        q[tail++] = sr * cols + sc;
        while (head < tail) {
            const int u = q[head++];
            const int ur = u / cols, uc = u % cols;
            const int nb[4][2] = {{ur - 1, uc}, {ur + 1, uc}, {ur, uc - 1}, {ur, uc + 1}};
            for (int d = 0; d < 4; ++d) {
                if (!passable(obs, rows, cols, nb[d][0], nb[d][1])) continue;
                const int v = nb[d][0] * cols + nb[d][1];
                if (dist[v] == INF) {
                    dist[v] = add_d(dist[u], 1);
                    q[tail++] = v;
                }
            }
        }
        for (int j = 0; j < k; ++j) {
            const int r = vps[2 * j], c = vps[2 * j + 1];
            if (passable(obs, rows, cols, r, c)) out[(size_t)i * k + j] = dist[(size_t)r * cols + c];
        }
    }
    free(q);
    free(dist);
}
