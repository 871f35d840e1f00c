/*
 * dsx_oracle.c -- plain-C restatement of dsDecompX's Host-mode hot path for a
 * virtual grid of P subdomains.  TEST INFRASTRUCTURE ONLY (see dsx_oracle.h).
 *
 * The reference runs one MPI rank per subdomain; here the P ranks are plain
 * structs and every message the MPI backend would carry is a direct read of
 * the sending rank's buffer, with the same matching rule: a rank receives, for
 * its neighbor entry n, what that neighbor sent toward direction -d_n
 * (src/backends/mpi_backend.cpp:398-433, tags base+slot(d) / base+slot(-d)).
 *
 * Compile with -ffp-contract=off: every floating-point expression below must
 * round exactly like the reference's (which is built without FMA contraction).
 */
#include "dsx_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXN 26
#define MAXF 16

typedef struct {
    double x, y, z, vx, vy, vz, fx, fy, fz, mass, charge;
    int type, gid;
} rec_t;

typedef struct {
    size_t owned, ghosts, cap;
    double* d[11];
    int* type;
    int* gid;
    unsigned char* field[MAXF];
} parts_t;

typedef struct {
    int coords[3];
    double lo[3], hi[3];
    int nn;
    int nrank[MAXN];
    int dir[MAXN][3];
    int slot[MAXN];
    double shift[MAXN][3];
    /* host halo plan (src/halo.cpp:164-238) */
    int plan_valid;
    int* src[MAXN];
    size_t src_n[MAXN], src_cap[MAXN];
    rec_t* send[MAXN];
    size_t recv_n[MAXN];
    parts_t p;
} rank_t;

struct orc_grid {
    int P, dims[3], policy, edges, periodic[3], nfields;
    double lower[3], upper[3], halo;
    double dyn_threshold, dyn_relax, dyn_minfrac;
    size_t dyn_interval, migration_calls;
    int in_rebalance;
    double* next_work;   /* work of the next automatic rebalance (null: owned counts) */
    int ghosts_valid;
    int ftype[MAXF];
    size_t fcomp[MAXF], fbytes[MAXF];
    double* cuts[3];
    rank_t* r;
    char err[512];
};

static size_t type_size(int t) {
    switch (t) {
    case 0: case 2: case 4: return 4;
    case 1: case 3: case 5: return 8;
    default: return 0;
    }
}

static int fail(orc_grid* g, const char* msg) {
    snprintf(g->err, sizeof g->err, "%s", msg);
    return -1;
}

/* ---------------- particle storage ---------------- */

static void parts_reserve(orc_grid* g, parts_t* p, size_t need) {
    if (need <= p->cap) return;
    size_t cap = p->cap ? p->cap : 16;
    while (cap < need) cap += cap / 2 + 1;
    for (int a = 0; a < 11; ++a) p->d[a] = realloc(p->d[a], cap * sizeof(double));
    p->type = realloc(p->type, cap * sizeof(int));
    p->gid = realloc(p->gid, cap * sizeof(int));
    for (int f = 0; f < g->nfields; ++f) p->field[f] = realloc(p->field[f], cap * g->fbytes[f]);
    p->cap = cap;
}

static void parts_free(orc_grid* g, parts_t* p) {
    for (int a = 0; a < 11; ++a) free(p->d[a]);
    free(p->type);
    free(p->gid);
    for (int f = 0; f < g->nfields; ++f) free(p->field[f]);
    memset(p, 0, sizeof *p);
}

/* copy_record (src/runtime.cpp:82-96) */
static void put_record(parts_t* p, size_t i, const rec_t* r) {
    p->d[0][i] = r->x; p->d[1][i] = r->y; p->d[2][i] = r->z;
    p->d[3][i] = r->vx; p->d[4][i] = r->vy; p->d[5][i] = r->vz;
    p->d[6][i] = r->fx; p->d[7][i] = r->fy; p->d[8][i] = r->fz;
    p->d[9][i] = r->mass; p->d[10][i] = r->charge;
    p->type[i] = r->type; p->gid[i] = r->gid;
}

/* ---------------- topology (src/topology.cpp, src/grid.cpp) ------------- */

/* direction_slot (src/topology.cpp:11-14) */
static int direction_slot(int dx, int dy, int dz) {
    int raw = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
    return raw < 13 ? raw : raw - 1;
}

/* MPI row-major Cartesian ranks, as MPI_Cart_rank/MPI_Cart_coords number them */
static int cart_rank(const orc_grid* g, const int* c) {
    return (c[0] * g->dims[1] + c[1]) * g->dims[2] + c[2];
}

/* balanced_score (src/grid.cpp:12-22) */
static double balanced_score(const int* grid, const double* len) {
    double lx = len[0] / grid[0], ly = len[1] / grid[1], lz = len[2] / grid[2];
    double stv = 2.0 * (1.0 / lx + 1.0 / ly + 1.0 / lz);
    double longest = lx, shortest = lx;
    if (ly > longest) longest = ly;
    if (lz > longest) longest = lz;
    if (ly < shortest) shortest = ly;
    if (lz < shortest) shortest = lz;
    double aspect = log(longest / shortest);
    return stv * (1.0 + 0.05 * aspect);
}

/* topology_score (src/grid.cpp:28-75) with every rank on one node, which is
 * what topology discovery reports when all ranks share a host
 * (src/backends/mpi_backend.cpp:898-947) */
static double topology_score(const int* grid, const double* len, const int* periodic) {
    double local[3] = {len[0] / grid[0], len[1] / grid[1], len[2] / grid[2]};
    double face[3] = {local[1] * local[2], local[0] * local[2], local[0] * local[1]};
    double cost = 0.0;
    for (int x = 0; x < grid[0]; ++x)
        for (int y = 0; y < grid[1]; ++y)
            for (int z = 0; z < grid[2]; ++z) {
                int source = (x * grid[1] + y) * grid[2] + z;
                for (int axis = 0; axis < 3; ++axis) {
                    int nc[3] = {x, y, z};
                    ++nc[axis];
                    if (nc[axis] == grid[axis]) {
                        if (!periodic[axis] || grid[axis] == 1) continue;
                        nc[axis] = 0;
                    }
                    int peer = (nc[0] * grid[1] + nc[1]) * grid[2] + nc[2];
                    if (peer == source) continue;
                    cost += face[axis] * 1.0;
                }
            }
    double volume = local[0] * local[1] * local[2];
    return cost / (volume * grid[0] * grid[1] * grid[2]) + 0.01 * balanced_score(grid, len);
}

/* choose_process_grid (src/grid.cpp:79-122), non-Manual policies */
static void choose_grid(int n, const double* len, const int* periodic, int policy, int* out) {
    double best_score = INFINITY;
    int best[3] = {n, 1, 1};
    for (int px = 1; px <= n; ++px) {
        if (n % px) continue;
        int remaining = n / px;
        for (int py = 1; py <= remaining; ++py) {
            if (remaining % py) continue;
            int cand[3] = {px, py, remaining / py};
            double score = policy == 2 ? topology_score(cand, len, periodic)
                                       : balanced_score(cand, len);
            /* lexicographic (score, px, py, pz) < (best_score, ...) */
            int less = 0;
            if (score < best_score) less = 1;
            else if (!(best_score < score)) {
                if (cand[0] != best[0]) less = cand[0] < best[0];
                else if (cand[1] != best[1]) less = cand[1] < best[1];
                else less = cand[2] < best[2];
            }
            if (less) {
                best_score = score;
                best[0] = cand[0]; best[1] = cand[1]; best[2] = cand[2];
            }
        }
    }
    out[0] = best[0]; out[1] = best[1]; out[2] = best[2];
}

/* MPI_Dims_create as the in-process MPI stand-in implements it */
static int dims_create(int n, int* dims) {
    int fixed = 1, free_count = 0;
    for (int d = 0; d < 3; ++d) {
        if (dims[d] > 0) fixed *= dims[d];
        else ++free_count;
    }
    if (free_count == 0) return fixed == n ? 0 : -1;
    if (n % fixed) return -1;
    int rem = n / fixed, factors[64], nf = 0;
    for (int f = 2; rem > 1 && f * f <= rem; ++f)
        while (rem % f == 0) { factors[nf++] = f; rem /= f; }
    if (rem > 1) factors[nf++] = rem;
    /* largest factor first */
    for (int i = 0; i < nf; ++i)
        for (int j = i + 1; j < nf; ++j)
            if (factors[j] > factors[i]) { int t = factors[i]; factors[i] = factors[j]; factors[j] = t; }
    int grid[3] = {1, 1, 1};
    for (int i = 0; i < nf; ++i) {
        int k = 0;
        for (int j = 1; j < free_count; ++j) if (grid[j] < grid[k]) k = j;
        grid[k] *= factors[i];
    }
    for (int i = 0; i < free_count; ++i)
        for (int j = i + 1; j < free_count; ++j)
            if (grid[j] > grid[i]) { int t = grid[i]; grid[i] = grid[j]; grid[j] = t; }
    int next = 0;
    for (int d = 0; d < 3; ++d) if (dims[d] <= 0) dims[d] = grid[next++];
    return 0;
}

/* refresh_domain_geometry (src/topology.cpp:57-176), for every rank */
static void refresh_geometry(orc_grid* g) {
    for (int s = 0; s < g->P; ++s) {
        rank_t* r = &g->r[s];
        int c[3];
        c[2] = s % g->dims[2];
        c[1] = (s / g->dims[2]) % g->dims[1];
        c[0] = s / (g->dims[1] * g->dims[2]);
        for (int a = 0; a < 3; ++a) {
            r->coords[a] = c[a];
            r->lo[a] = g->cuts[a][c[a]];
            r->hi[a] = g->cuts[a][c[a] + 1];
        }
        r->nn = 0;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    if (!dx && !dy && !dz) continue;
                    if (!g->edges && abs(dx) + abs(dy) + abs(dz) != 1) continue;
                    int d[3] = {dx, dy, dz};
                    int touches = 0;
                    for (int a = 0; a < 3; ++a) if (d[a] != 0 && g->dims[a] == 1) touches = 1;
                    if (touches) continue;
                    int nc[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
                    double shift[3] = {0.0, 0.0, 0.0};
                    int outside = 0;
                    for (int a = 0; a < 3; ++a) {
                        if (nc[a] < 0 || nc[a] >= g->dims[a]) {
                            if (!g->periodic[a]) { outside = 1; break; }
                            double extent = g->upper[a] - g->lower[a];
                            if (nc[a] < 0) { nc[a] += g->dims[a]; shift[a] = extent; }
                            else { nc[a] -= g->dims[a]; shift[a] = -extent; }
                        }
                    }
                    int n = r->nn++;
                    r->dir[n][0] = dx; r->dir[n][1] = dy; r->dir[n][2] = dz;
                    for (int a = 0; a < 3; ++a) r->shift[n][a] = shift[a];
                    r->slot[n] = direction_slot(dx, dy, dz);
                    r->nrank[n] = outside ? -1 : cart_rank(g, nc);
                }
        r->plan_valid = 0;
    }
}

/* uniform cuts (src/topology.cpp:63-75) */
static void uniform_cuts(orc_grid* g) {
    for (int a = 0; a < 3; ++a) {
        free(g->cuts[a]);
        g->cuts[a] = malloc(sizeof(double) * (size_t)(g->dims[a] + 1));
        double extent = g->upper[a] - g->lower[a];
        for (int i = 0; i <= g->dims[a]; ++i)
            g->cuts[a][i] = g->lower[a] + extent * (double)i / (double)g->dims[a];
    }
}

/* Periodic wrap of Decomposition::owner_rank and wrapped_record
 * (src/migration.cpp:83-87, 106-113) */
static double wrap_axis(const orc_grid* g, double v, int a) {
    if (!g->periodic[a]) return v;
    double lower = g->lower[a];
    double extent = g->upper[a] - lower;
    v -= lower;
    v -= floor(v / extent) * extent;
    return v + lower;
}

/* std::upper_bound(cuts, value) - 1, clamped (src/migration.cpp:89-93) */
static int axis_coordinate(const orc_grid* g, double v, int a) {
    int lo = 0, hi = g->dims[a] + 1;
    while (lo < hi) {
        int mid = lo + (hi - lo) / 2;
        if (v < g->cuts[a][mid]) hi = mid;
        else lo = mid + 1;
    }
    int c = lo - 1;
    if (c > g->dims[a] - 1) c = g->dims[a] - 1;
    if (c < 0) c = 0;
    return c;
}

/* Decomposition::owner_rank (src/migration.cpp:74-98) */
static int owner_rank(const orc_grid* g, double x, double y, double z) {
    double p[3] = {x, y, z};
    int c[3];
    for (int a = 0; a < 3; ++a) c[a] = axis_coordinate(g, wrap_axis(g, p[a], a), a);
    return cart_rank(g, c);
}

/* ---------------- create / destroy ---------------- */

orc_grid* orc_create(int nranks, const int* dims, int policy, const double* lower,
                     const double* upper, const int* periodic, double halo_width,
                     int edges_and_corners, const double* dynamic, int nfields,
                     const int* types, const long long* components, char* error,
                     int error_length) {
    char msg[256] = "";
    if (nranks <= 0) snprintf(msg, sizeof msg, "nranks must be positive");
    for (int a = 0; a < 3 && !msg[0]; ++a)
        if (!(upper[a] > lower[a])) snprintf(msg, sizeof msg, "global-domain extent must be positive");
    if (!msg[0] && halo_width < 0.0) snprintf(msg, sizeof msg, "halo width cannot be negative");
    if (!msg[0] && (nfields < 0 || nfields > MAXF)) snprintf(msg, sizeof msg, "too many fields");
    if (!msg[0] && dynamic &&
        (!(dynamic[1] >= 1.0) || !(dynamic[2] > 0.0 && dynamic[2] <= 1.0) ||
         !(dynamic[3] > 0.0 && dynamic[3] <= 1.0)))
        snprintf(msg, sizeof msg, "invalid dynamic load-balance configuration");
    orc_grid* g = NULL;
    if (!msg[0]) {
        g = calloc(1, sizeof *g);
        g->P = nranks;
        g->policy = policy;
        g->edges = edges_and_corners;
        g->halo = halo_width;
        for (int a = 0; a < 3; ++a) {
            g->lower[a] = lower[a];
            g->upper[a] = upper[a];
            g->periodic[a] = periodic[a] != 0;
        }
        g->dyn_interval = dynamic ? (size_t)dynamic[0] : 1;
        g->dyn_threshold = dynamic ? dynamic[1] : 1.10;
        g->dyn_relax = dynamic ? dynamic[2] : 0.5;
        g->dyn_minfrac = dynamic ? dynamic[3] : 0.10;
        g->nfields = nfields;
        for (int f = 0; f < nfields; ++f) {
            g->ftype[f] = types[f];
            g->fcomp[f] = (size_t)components[f];
            g->fbytes[f] = g->fcomp[f] * type_size(types[f]);
        }
        /* initialize_topology (src/topology.cpp:18-55) */
        if (policy != 0) {
            double len[3] = {upper[0] - lower[0], upper[1] - lower[1], upper[2] - lower[2]};
            choose_grid(nranks, len, g->periodic, policy, g->dims);
        } else {
            for (int a = 0; a < 3; ++a) g->dims[a] = dims[a];
            for (int a = 0; a < 3 && !msg[0]; ++a)
                if (dims[a] < 0) snprintf(msg, sizeof msg, "process-grid dimensions cannot be negative");
        }
        if (!msg[0] && dims_create(nranks, g->dims) != 0)
            snprintf(msg, sizeof msg, "process-grid dimensions do not match communicator size");
    }
    if (msg[0]) {
        if (error && error_length > 0) snprintf(error, (size_t)error_length, "%s", msg);
        free(g);
        return NULL;
    }
    g->r = calloc((size_t)nranks, sizeof(rank_t));
    uniform_cuts(g);
    refresh_geometry(g);
    return g;
}

void orc_destroy(orc_grid* g) {
    if (!g) return;
    for (int s = 0; s < g->P; ++s) {
        rank_t* r = &g->r[s];
        for (int n = 0; n < MAXN; ++n) { free(r->src[n]); free(r->send[n]); }
        parts_free(g, &r->p);
    }
    free(g->r);
    for (int a = 0; a < 3; ++a) free(g->cuts[a]);
    free(g->next_work);
    free(g);
}

/* Work per rank for the next migrate's automatic rebalance instead of the
 * owned counts (a sharded run passes the counts of every shard). */
int orc_set_rebalance_work(orc_grid* g, const double* work) {
    free(g->next_work);
    g->next_work = NULL;
    if (!work) return 0;
    g->next_work = malloc(sizeof(double) * (size_t)g->P);
    memcpy(g->next_work, work, sizeof(double) * (size_t)g->P);
    return 0;
}

const char* orc_last_error(orc_grid* g) { return g ? g->err : "null grid"; }
int orc_size(orc_grid* g) { return g->P; }

int orc_topology(orc_grid* g, int rank, int* dims, int* coords, double* local) {
    rank_t* r = &g->r[rank];
    for (int a = 0; a < 3; ++a) {
        dims[a] = g->dims[a];
        coords[a] = r->coords[a];
        local[a] = r->lo[a];
        local[3 + a] = r->hi[a];
    }
    return 0;
}

int orc_neighbors(orc_grid* g, int rank, int* count, int* info, double* shifts) {
    rank_t* r = &g->r[rank];
    *count = r->nn;
    for (int n = 0; n < r->nn; ++n) {
        info[5 * n + 0] = r->nrank[n];
        info[5 * n + 1] = r->dir[n][0];
        info[5 * n + 2] = r->dir[n][1];
        info[5 * n + 3] = r->dir[n][2];
        info[5 * n + 4] = r->slot[n];
        for (int a = 0; a < 3; ++a) shifts[3 * n + a] = r->shift[n][a];
    }
    return 0;
}

int orc_cuts(orc_grid* g, double* out) {
    size_t k = 0;
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i <= g->dims[a]; ++i) out[k++] = g->cuts[a][i];
    return 0;
}

int orc_owner_rank(orc_grid* g, long long n, const double* pos, int* out) {
    for (long long i = 0; i < n; ++i) out[i] = owner_rank(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    return 0;
}

/* ---------------- particle access ---------------- */

int orc_set_owned(orc_grid* g, int rank, long long n, const double* const* core,
                  const int* type, const int* gid, const void* const* fields) {
    rank_t* r = &g->r[rank];
    parts_t* p = &r->p;
    parts_reserve(g, p, (size_t)n);
    for (int a = 0; a < 11; ++a) {
        if (core && core[a]) memcpy(p->d[a], core[a], sizeof(double) * (size_t)n);
        else memset(p->d[a], 0, sizeof(double) * (size_t)n);
    }
    if (type) memcpy(p->type, type, sizeof(int) * (size_t)n);
    else memset(p->type, 0, sizeof(int) * (size_t)n);
    if (gid) memcpy(p->gid, gid, sizeof(int) * (size_t)n);
    else memset(p->gid, 0, sizeof(int) * (size_t)n);
    for (int f = 0; f < g->nfields; ++f) {
        if (fields && fields[f]) memcpy(p->field[f], fields[f], g->fbytes[f] * (size_t)n);
        else memset(p->field[f], 0, g->fbytes[f] * (size_t)n);
    }
    p->owned = (size_t)n;
    p->ghosts = 0;
    return 0;
}

/* Ghosts of rank `rank` per receive block m (its neighbor order), as the
 * last exchange_halo laid them out: out[m] for m < *count. */
int orc_halo_blocks(orc_grid* g, int rank, int* count, long long* out) {
    const rank_t* r = &g->r[rank];
    *count = r->nn;
    for (int m = 0; m < r->nn; ++m) out[m] = g->ghosts_valid ? (long long)r->recv_n[m] : 0;
    return 0;
}

int orc_counts(orc_grid* g, int rank, long long* owned, long long* ghosts) {
    *owned = (long long)g->r[rank].p.owned;
    *ghosts = (long long)g->r[rank].p.ghosts;
    return 0;
}

static unsigned char* array_base(orc_grid* g, parts_t* p, int array, size_t* element) {
    if (array >= 0 && array <= 10) { *element = 8; return (unsigned char*)p->d[array]; }
    if (array == 11) { *element = 4; return (unsigned char*)p->type; }
    if (array == 12) { *element = 4; return (unsigned char*)p->gid; }
    int f = array - 13;
    if (f < 0 || f >= g->nfields) return NULL;
    *element = g->fbytes[f];
    return p->field[f];
}

int orc_read(orc_grid* g, int rank, int array, long long start, long long count, void* out) {
    parts_t* p = &g->r[rank].p;
    size_t element = 0;
    unsigned char* base = array_base(g, p, array, &element);
    if (!base && count) return fail(g, "bad array id");
    if ((size_t)(start + count) > p->owned + p->ghosts) return fail(g, "read past the particle count");
    if (count) memcpy(out, base + element * (size_t)start, element * (size_t)count);
    return 0;
}

int orc_write(orc_grid* g, int rank, int array, long long start, long long count, const void* in) {
    parts_t* p = &g->r[rank].p;
    size_t element = 0;
    unsigned char* base = array_base(g, p, array, &element);
    if (!base && count) return fail(g, "bad array id");
    if ((size_t)(start + count) > p->owned + p->ghosts) return fail(g, "write past the particle count");
    if (count) memcpy(base + element * (size_t)start, in, element * (size_t)count);
    return 0;
}

/* ---------------- dynamic rebalance (src/runtime.cpp:345-447) ------------ */

static int set_axis_cuts(orc_grid* g, double* const* cuts);

static int rebalance_geometry(orc_grid* g, const double* work, int force, int* attempted,
                              int* changed, double* imbalance) {
    for (int s = 0; s < g->P; ++s)
        if (!isfinite(work[s]) || work[s] < 0.0)
            return fail(g, "rebalance local_work must be finite and non-negative");
    double total = 0.0, maximum = 0.0;
    for (int s = 0; s < g->P; ++s) {
        total += work[s];
        if (maximum < work[s]) maximum = work[s];
    }
    *attempted = 1;
    *changed = 0;
    *imbalance = 1.0;
    if (total <= 0.0 || g->P <= 1) return 0;
    *imbalance = maximum / (total / (double)g->P);
    if (!force && *imbalance < g->dyn_threshold) return 0;

    double* cuts[3];
    for (int a = 0; a < 3; ++a) {
        cuts[a] = malloc(sizeof(double) * (size_t)(g->dims[a] + 1));
        memcpy(cuts[a], g->cuts[a], sizeof(double) * (size_t)(g->dims[a] + 1));
    }
    for (int a = 0; a < 3; ++a) {
        int slabs = g->dims[a];
        if (slabs <= 1) continue;
        double* slab_work = calloc((size_t)slabs, sizeof(double));
        for (int s = 0; s < g->P; ++s) slab_work[g->r[s].coords[a]] += work[s];
        double* old_cuts = malloc(sizeof(double) * (size_t)(slabs + 1));
        memcpy(old_cuts, cuts[a], sizeof(double) * (size_t)(slabs + 1));
        double target = total / (double)slabs;
        double extent = g->upper[a] - g->lower[a];
        double uniform = extent / (double)slabs;
        double lower_bound = uniform * g->dyn_minfrac;
        if (lower_bound < g->halo) lower_bound = g->halo;          /* std::max */
        double minimum_width = lower_bound < uniform ? lower_bound : uniform; /* std::min */
        cuts[a][0] = g->lower[a];
        cuts[a][slabs] = g->upper[a];
        for (int b = 1; b < slabs; ++b) {
            double desired = target * (double)b;
            double cumulative = 0.0;
            int slab = 0;
            while (slab < slabs - 1 && cumulative + slab_work[slab] < desired)
                cumulative += slab_work[slab++];
            double weight = slab_work[slab];
            double fraction;
            if (weight > 0.0) {
                double v = (desired - cumulative) / weight;
                fraction = v < 0.0 ? 0.0 : (1.0 < v ? 1.0 : v);   /* std::clamp */
            } else {
                fraction = 0.5;
            }
            double proposed = old_cuts[slab] + fraction * (old_cuts[slab + 1] - old_cuts[slab]);
            double old = old_cuts[b];
            cuts[a][b] = old + g->dyn_relax * (proposed - old);
        }
        for (int i = 1; i < slabs; ++i) {
            double floor_value = cuts[a][i - 1] + minimum_width;
            if (cuts[a][i] < floor_value) cuts[a][i] = floor_value;
        }
        for (int i = slabs - 1; i > 0; --i) {
            double ceiling = cuts[a][i + 1] - minimum_width;
            if (ceiling < cuts[a][i]) cuts[a][i] = ceiling;
        }
        free(slab_work);
        free(old_cuts);
    }
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i <= g->dims[a]; ++i)
            if (fabs(cuts[a][i] - g->cuts[a][i]) > 1.0e-12) *changed = 1;
    int status = 0;
    if (*changed) status = set_axis_cuts(g, cuts);
    for (int a = 0; a < 3; ++a) free(cuts[a]);
    return status;
}

/* Decomposition::set_axis_cuts (src/decomp.cpp:146-163) */
static int set_axis_cuts(orc_grid* g, double* const* cuts) {
    for (int a = 0; a < 3; ++a) {
        int n = g->dims[a];
        if (cuts[a][0] != g->lower[a] || cuts[a][n] != g->upper[a])
            return fail(g, "dynamic cuts must be strictly increasing and span the domain");
        for (int i = 0; i < n; ++i)
            if (!(cuts[a][i] < cuts[a][i + 1]))
                return fail(g, "dynamic cuts must be strictly increasing and span the domain");
    }
    for (int a = 0; a < 3; ++a)
        memcpy(g->cuts[a], cuts[a], sizeof(double) * (size_t)(g->dims[a] + 1));
    refresh_geometry(g);
    return 0;
}

/* ---------------- migrate (src/migration.cpp:395-591) ---------------- */

static rec_t wrapped_record(const orc_grid* g, const parts_t* p, size_t i) {
    rec_t r;
    r.x = wrap_axis(g, p->d[0][i], 0);
    r.y = wrap_axis(g, p->d[1][i], 1);
    r.z = wrap_axis(g, p->d[2][i], 2);
    r.vx = p->d[3][i]; r.vy = p->d[4][i]; r.vz = p->d[5][i];
    r.fx = p->d[6][i]; r.fy = p->d[7][i]; r.fz = p->d[8][i];
    r.mass = p->d[9][i]; r.charge = p->d[10][i];
    r.type = p->type[i];
    r.gid = p->gid[i];
    return r;
}

static int migrate_inner(orc_grid* g, long long* results) {
    /* Decomp::migrate (src/runtime.cpp:983-1019): automatic Dynamic rebalance */
    ++g->migration_calls;
    double* supplied = g->next_work;   /* one migrate only */
    g->next_work = NULL;
    if (!g->in_rebalance && g->policy == 3 && g->dyn_interval != 0 &&
        g->migration_calls % g->dyn_interval == 0) {
        double* work = malloc(sizeof(double) * (size_t)g->P);
        for (int s = 0; s < g->P; ++s)
            work[s] = supplied ? supplied[s] : (double)g->r[s].p.owned;
        int attempted, changed;
        double imbalance;
        int status = rebalance_geometry(g, work, 0, &attempted, &changed, &imbalance);
        free(work);
        if (status) {
            free(supplied);
            return status;
        }
    }
    free(supplied);
    int P = g->P;
    /* classify (src/migration.cpp:437-445) */
    int** dest = malloc(sizeof(int*) * (size_t)P);
    size_t* retained = calloc((size_t)P, sizeof(size_t));
    size_t* received = calloc((size_t)P, sizeof(size_t));
    for (int s = 0; s < P; ++s) {
        parts_t* p = &g->r[s].p;
        dest[s] = malloc(sizeof(int) * (p->owned ? p->owned : 1));
        for (size_t i = 0; i < p->owned; ++i) {
            rec_t rec = wrapped_record(g, p, i);
            int d = owner_rank(g, rec.x, rec.y, rec.z);
            dest[s][i] = d;
            if (d == s) ++retained[s];
            else ++received[d];
        }
    }
    /* pack + compact: retained in original order, then what each peer sent,
     * peers in rank order (src/migration.cpp:458-518) */
    parts_t* next = calloc((size_t)P, sizeof(parts_t));
    for (int d = 0; d < P; ++d) {
        size_t total = retained[d] + received[d];
        parts_reserve(g, &next[d], total ? total : 1);
        size_t k = 0;
        for (int pass = 0; pass <= P; ++pass) {
            /* pass 0: d's own retained particles; pass 1+s: arrivals from s */
            int s = pass == 0 ? d : pass - 1;
            if (pass > 0 && s == d) continue;
            parts_t* p = &g->r[s].p;
            for (size_t i = 0; i < p->owned; ++i) {
                if (dest[s][i] != d) continue;
                rec_t rec = wrapped_record(g, p, i);
                put_record(&next[d], k, &rec);
                for (int f = 0; f < g->nfields; ++f)
                    memcpy(next[d].field[f] + k * g->fbytes[f], p->field[f] + i * g->fbytes[f], g->fbytes[f]);
                ++k;
            }
        }
        next[d].owned = total;
        next[d].ghosts = 0;
    }
    for (int s = 0; s < P; ++s) {
        parts_t* p = &g->r[s].p;
        if (results) {
            long long* o = results + 6 * s;
            o[1] = (long long)p->owned;
            o[2] = (long long)retained[s];
            o[3] = (long long)(p->owned - retained[s]);
            o[4] = (long long)received[s];
            o[5] = (long long)(retained[s] + received[s]);
            o[0] = (o[3] != 0 || o[4] != 0);
        }
    }
    for (int s = 0; s < P; ++s) {
        parts_free(g, &g->r[s].p);
        g->r[s].p = next[s];
        g->r[s].plan_valid = 0;   /* invalidate_halo_plan (src/migration.cpp:590) */
        free(dest[s]);
    }
    g->ghosts_valid = 0;
    free(next);
    free(dest);
    free(retained);
    free(received);
    return 0;
}

int orc_migrate(orc_grid* g, long long* results) { return migrate_inner(g, results); }

/* Decomp::rebalance (src/runtime.cpp:1021-1041) */
int orc_rebalance(orc_grid* g, const double* local_work, int force, long long* results,
                  double* imbalance) {
    double* work = malloc(sizeof(double) * (size_t)g->P);
    for (int s = 0; s < g->P; ++s)
        work[s] = local_work && local_work[s] >= 0.0 ? local_work[s] : (double)g->r[s].p.owned;
    int attempted = 0, changed = 0;
    double imb = 1.0;
    int status = rebalance_geometry(g, work, force, &attempted, &changed, &imb);
    free(work);
    if (status) return status;
    long long* mig = malloc(sizeof(long long) * 6 * (size_t)g->P);
    g->in_rebalance = 1;
    status = migrate_inner(g, mig);
    g->in_rebalance = 0;
    for (int s = 0; s < g->P && status == 0; ++s) {
        if (results) {
            results[3 * s + 0] = attempted;
            results[3 * s + 1] = changed;
            results[3 * s + 2] = mig[6 * s + 5];
        }
        if (imbalance) imbalance[s] = imb;
    }
    free(mig);
    return status;
}

int orc_set_halo_width(orc_grid* g, double width) {
    if (width < 0.0) return fail(g, "halo width cannot be negative");
    if (g->halo != width) {
        g->halo = width;
        for (int s = 0; s < g->P; ++s) g->r[s].plan_valid = 0;
    }
    return 0;
}

int orc_invalidate_halo(orc_grid* g) {
    for (int s = 0; s < g->P; ++s) g->r[s].plan_valid = 0;
    return 0;
}

/* Decomposition::set_axis_cuts (dsDecompX src/decomp.cpp:146-163): the cuts
   must span the domain and increase strictly; the geometry is refreshed and
   the halo plan invalid. */
int orc_set_cuts(orc_grid* g, const double* cuts) {
    int off = 0;
    for (int a = 0; a < 3; ++a) {
        const double* c = cuts + off;
        int ok = c[0] == g->lower[a] && c[g->dims[a]] == g->upper[a];
        for (int i = 0; i < g->dims[a]; ++i) ok = ok && c[i] < c[i + 1];
        if (!ok) return fail(g, "dynamic cuts must be strictly increasing and span the domain");
        off += g->dims[a] + 1;
    }
    off = 0;
    for (int a = 0; a < 3; ++a) {
        for (int i = 0; i <= g->dims[a]; ++i) g->cuts[a][i] = cuts[off + i];
        off += g->dims[a] + 1;
    }
    refresh_geometry(g);
    return 0;
}

/* Decomposition::rescale_domain / update_domain (dsDecompX
   src/decomp.cpp:104-144): every cut keeps its fraction of the extent, the
   neighbours' periodic shifts follow the new extent; rescale keeps the halo
   plan (same grid, same neighbours), update invalidates it.  Positions are
   the caller's. */
int orc_rescale_domain(orc_grid* g, const double* lower, const double* upper, int invalidate) {
    for (int a = 0; a < 3; ++a) {
        const double old_extent = g->upper[a] - g->lower[a];
        const double new_extent = upper[a] - lower[a];
        for (int i = 0; i <= g->dims[a]; ++i) {
            const double fraction = (g->cuts[a][i] - g->lower[a]) / old_extent;
            g->cuts[a][i] = lower[a] + fraction * new_extent;
        }
    }
    for (int a = 0; a < 3; ++a) {
        g->lower[a] = lower[a];
        g->upper[a] = upper[a];
    }
    int* valid = malloc(sizeof(int) * (size_t)g->P);
    for (int s = 0; s < g->P; ++s) valid[s] = g->r[s].plan_valid;
    refresh_geometry(g);
    if (!invalidate)
        for (int s = 0; s < g->P; ++s) g->r[s].plan_valid = valid[s];
    free(valid);
    return 0;
}

/* ---------------- halo (src/halo.cpp) ---------------- */

static void plan_push(rank_t* r, int n, int index, const rec_t* rec) {
    if (r->src_n[n] == r->src_cap[n]) {
        size_t cap = r->src_cap[n] ? r->src_cap[n] + r->src_cap[n] / 2 + 1 : 64;
        r->src[n] = realloc(r->src[n], sizeof(int) * cap);
        r->send[n] = realloc(r->send[n], sizeof(rec_t) * cap);
        r->src_cap[n] = cap;
    }
    r->src[n][r->src_n[n]] = index;
    r->send[n][r->src_n[n]] = *rec;
    ++r->src_n[n];
}

/* rebuild_halo_plan (src/halo.cpp:164-238) with make_record (:37-55) */
static void rebuild_plan(orc_grid* g, rank_t* r) {
    const parts_t* p = &r->p;
    double w = g->halo;
    for (int n = 0; n < r->nn; ++n) { r->src_n[n] = 0; r->recv_n[n] = 0; }
    for (size_t i = 0; i < p->owned; ++i) {
        double px = p->d[0][i], py = p->d[1][i], pz = p->d[2][i];
        int xlo = px < r->lo[0] + w, xhi = px > r->hi[0] - w;
        int ylo = py < r->lo[1] + w, yhi = py > r->hi[1] - w;
        int zlo = pz < r->lo[2] + w, zhi = pz > r->hi[2] - w;
        if (!xlo && !xhi && !ylo && !yhi && !zlo && !zhi) continue;
        for (int n = 0; n < r->nn; ++n) {
            if (r->nrank[n] < 0) continue;
            if (r->dir[n][0] < 0 && !xlo) continue;
            if (r->dir[n][0] > 0 && !xhi) continue;
            if (r->dir[n][1] < 0 && !ylo) continue;
            if (r->dir[n][1] > 0 && !yhi) continue;
            if (r->dir[n][2] < 0 && !zlo) continue;
            if (r->dir[n][2] > 0 && !zhi) continue;
            rec_t rec;
            rec.x = p->d[0][i] + r->shift[n][0];
            rec.y = p->d[1][i] + r->shift[n][1];
            rec.z = p->d[2][i] + r->shift[n][2];
            rec.vx = p->d[3][i]; rec.vy = p->d[4][i]; rec.vz = p->d[5][i];
            rec.fx = 0.0; rec.fy = 0.0; rec.fz = 0.0;
            rec.mass = p->d[9][i]; rec.charge = p->d[10][i];
            rec.type = p->type[i];
            rec.gid = p->gid[i];
            plan_push(r, n, (int)i, &rec);
        }
    }
    r->plan_valid = 1;
}

/* refresh_halo_buffers (src/halo.cpp:256-289) */
static void refresh_plan(orc_grid* g, rank_t* r) {
    if (!r->plan_valid) { rebuild_plan(g, r); return; }
    const parts_t* p = &r->p;
    for (int n = 0; n < r->nn; ++n) {
        for (size_t k = 0; k < r->src_n[n]; ++k) {
            int i = r->src[n][k];
            if (i < 0 || (size_t)i >= p->owned) { rebuild_plan(g, r); return; }
            rec_t* rec = &r->send[n][k];
            rec->x = p->d[0][i] + r->shift[n][0];
            rec->y = p->d[1][i] + r->shift[n][1];
            rec->z = p->d[2][i] + r->shift[n][2];
            rec->vx = p->d[3][i]; rec->vy = p->d[4][i]; rec->vz = p->d[5][i];
        }
    }
}

/* The neighbor entry of rank `s` that sends toward direction -dir: the MPI
 * backend matches a receive on tag base+slot(-d_n) (mpi_backend.cpp:398-403). */
static int sender_entry(const orc_grid* g, int s, const int* dir) {
    const rank_t* r = &g->r[s];
    int want = direction_slot(-dir[0], -dir[1], -dir[2]);
    for (int n = 0; n < r->nn; ++n) if (r->slot[n] == want) return n;
    return -1;
}

int orc_exchange_halo(orc_grid* g, int rebuild, long long* results) {
    int P = g->P;
    if (rebuild) orc_invalidate_halo(g);
    /* previous ghost ids (src/runtime.cpp:900-905) */
    int** previous = calloc((size_t)P, sizeof(int*));
    size_t* previous_count = calloc((size_t)P, sizeof(size_t));
    for (int s = 0; s < P; ++s) {
        parts_t* p = &g->r[s].p;
        previous_count[s] = p->ghosts;
        if (p->ghosts) {
            previous[s] = malloc(sizeof(int) * p->ghosts);
            memcpy(previous[s], p->gid + p->owned, sizeof(int) * p->ghosts);
        }
    }
    if (P == 1) {
        /* one rank owns the whole periodic box: no ghosts (src/halo.cpp:325-350) */
        rank_t* r = &g->r[0];
        for (int n = 0; n < r->nn; ++n) { r->src_n[n] = 0; r->recv_n[n] = 0; }
        r->plan_valid = 0;
        r->p.ghosts = 0;
    } else {
        for (int s = 0; s < P; ++s) refresh_plan(g, &g->r[s]);
        /* receive: block m of rank q is what nbr(q,m) sent toward -d_m, in the
         * sender's order (src/halo.cpp:609-649; src/runtime.cpp:951-957) */
        for (int q = 0; q < P; ++q) {
            rank_t* r = &g->r[q];
            size_t total = 0;
            for (int m = 0; m < r->nn; ++m) {
                r->recv_n[m] = 0;
                int sender = r->nrank[m];
                if (sender < 0) continue;
                int e = sender_entry(g, sender, r->dir[m]);
                if (e >= 0) r->recv_n[m] = g->r[sender].src_n[e];
                total += r->recv_n[m];
            }
            parts_reserve(g, &r->p, r->p.owned + total);
            size_t slot = r->p.owned;
            for (int m = 0; m < r->nn; ++m) {
                if (!r->recv_n[m]) continue;
                int sender = r->nrank[m];
                const rank_t* sr = &g->r[sender];
                int e = sender_entry(g, sender, r->dir[m]);
                for (size_t k = 0; k < r->recv_n[m]; ++k, ++slot) {
                    put_record(&r->p, slot, &sr->send[e][k]);
                    /* pack_halo_fields: current field values of the source
                     * indices, every exchange (src/halo.cpp:120-147,687) */
                    size_t i = (size_t)sr->src[e][k];
                    for (int f = 0; f < g->nfields; ++f)
                        memcpy(r->p.field[f] + slot * g->fbytes[f], sr->p.field[f] + i * g->fbytes[f],
                               g->fbytes[f]);
                }
            }
            r->p.ghosts = total;
        }
    }
    for (int s = 0; s < P; ++s) {
        parts_t* p = &g->r[s].p;
        if (results) {
            /* layout_changed (src/runtime.cpp:966-980) */
            int changed = rebuild || previous_count[s] != p->ghosts;
            for (size_t i = 0; !changed && i < p->ghosts; ++i)
                if (previous[s][i] != p->gid[p->owned + i]) changed = 1;
            long long* o = results + 4 * s;
            o[0] = (long long)p->ghosts;
            o[1] = changed;
            o[2] = 0;
            o[3] = 0;
        }
        free(previous[s]);
    }
    free(previous);
    free(previous_count);
    g->ghosts_valid = P > 1;
    return 0;
}

/* reduce_field_values (src/halo.cpp:1351-1372): std::min / std::max /
 * += / = on the destination, ghosts taken in neighbor order n ascending and
 * plan order k (src/halo.cpp:1507-1530) */
#define REDUCE_CASE(T)                                                           \
    do {                                                                         \
        T* out = (T*)dst;                                                        \
        const T* in = (const T*)src;                                             \
        for (size_t c = 0; c < comps; ++c) {                                     \
            T v = in[c];                                                         \
            T* d = &out[c];                                                      \
            switch (op) {                                                        \
            case 0: *d = (T)(*d + v); break;                                     \
            case 1: if (v < *d) *d = v; break;                                   \
            case 2: if (*d < v) *d = v; break;                                   \
            default: *d = v; break;                                              \
            }                                                                    \
        }                                                                        \
    } while (0)

static void reduce_value(int type, int op, size_t comps, unsigned char* dst, const unsigned char* src) {
    switch (type) {
    case 0: REDUCE_CASE(int32_t); break;
    case 1: REDUCE_CASE(int64_t); break;
    case 2: REDUCE_CASE(uint32_t); break;
    case 3: REDUCE_CASE(uint64_t); break;
    case 4: REDUCE_CASE(float); break;
    default: REDUCE_CASE(double); break;
    }
}

/* Host reverse_exchange of one array (src/halo.cpp:1476-1531): rank r gets,
 * for its neighbor n, the ghost slice of block m at q = nbr(r,n) (the block q
 * received from r), and reduces it into src[n][k] in order. */
static void reverse_array(orc_grid* g, int array, int type, int op, size_t comps) {
    for (int s = 0; s < g->P; ++s) {
        rank_t* r = &g->r[s];
        size_t element = 0;
        unsigned char* owner_base = array_base(g, &r->p, array, &element);
        for (int n = 0; n < r->nn; ++n) {
            int q = r->nrank[n];
            if (q < 0 || r->src_n[n] == 0) continue;
            rank_t* rq = &g->r[q];
            int m = sender_entry(g, q, r->dir[n]);
            if (m < 0) continue;
            size_t offset = rq->p.owned;
            for (int mm = 0; mm < m; ++mm) offset += rq->recv_n[mm];
            size_t qe = 0;
            unsigned char* ghost_base = array_base(g, &rq->p, array, &qe);
            for (size_t k = 0; k < rq->recv_n[m] && k < r->src_n[n]; ++k)
                reduce_value(type, op, comps, owner_base + (size_t)r->src[n][k] * element,
                             ghost_base + (offset + k) * element);
        }
    }
}

/* Decomposition::reverse_halo on host memory: fx, fy, fz as Float64 Sum
 * (src/halo.cpp:1331-1346) */
int orc_reverse_halo(orc_grid* g) {
    if (g->P == 1 || !g->ghosts_valid) return 0;
    for (int a = 6; a <= 8; ++a) reverse_array(g, a, 5, 0, 1);
    return 0;
}

int orc_reverse_exchange(orc_grid* g, int nfields, const int* ids, const int* ops) {
    for (int i = 0; i < nfields; ++i)
        for (int j = i + 1; j < nfields; ++j)
            if (ids[i] == ids[j]) return fail(g, "duplicate reverse exchange field");
    for (int i = 0; i < nfields; ++i)
        if (ids[i] < 0 || ids[i] >= g->nfields) return fail(g, "missing or undersized reverse exchange field");
    if (g->P == 1 || !g->ghosts_valid) return 0;
    for (int i = 0; i < nfields; ++i)
        reverse_array(g, 13 + ids[i], g->ftype[ids[i]], ops[i], g->fcomp[ids[i]]);
    return 0;
}

/* forward field copy: every ghost slot gets its owner's current value along
 * the last halo plan -- the values a Host exchange_halo delivers for a field
 * (src/halo.cpp:120-147, 874-890); the CUDA forward_exchange's contract
 * (src/halo.cpp:1210-1286). */
int orc_forward_exchange(orc_grid* g, int nfields, const int* ids) {
    for (int i = 0; i < nfields; ++i)
        for (int j = i + 1; j < nfields; ++j)
            if (ids[i] == ids[j]) return fail(g, "duplicate forward exchange field");
    for (int i = 0; i < nfields; ++i)
        if (ids[i] < 0 || ids[i] >= g->nfields) return fail(g, "missing or undersized forward exchange field");
    if (g->P == 1 || !g->ghosts_valid) return 0;
    for (int q = 0; q < g->P; ++q) {
        rank_t* r = &g->r[q];
        size_t slot = r->p.owned;
        for (int m = 0; m < r->nn; ++m) {
            if (!r->recv_n[m]) continue;
            const rank_t* sr = &g->r[r->nrank[m]];
            int e = sender_entry(g, r->nrank[m], r->dir[m]);
            for (size_t k = 0; k < r->recv_n[m]; ++k, ++slot) {
                size_t i = (size_t)sr->src[e][k];
                for (int t = 0; t < nfields; ++t) {
                    int f = ids[t];
                    memcpy(r->p.field[f] + slot * g->fbytes[f], sr->p.field[f] + i * g->fbytes[f], g->fbytes[f]);
                }
            }
        }
    }
    return 0;
}
