/*
 * bh_oracle.c -- CPU oracle for the Barnes-Hut force path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; only the tests, the smoke check and the CPU-baseline leg of
 * the benchmark do, and only as the checker / the timed reference-equivalent
 * CPU code.
 *
 * This is a C restatement of the reference's Fortran (Potalej/hierarquicos),
 * written to keep the reference's operation order so that integer results
 * (Morton keys, sort permutation, node topology) are bit-exact and floating
 * point results differ from the Fortran only by rounding.  Every function
 * cites the reference file:line it follows.  Index conventions: the Fortran is
 * 1-based; here every particle / node index is 0-based and the Fortran
 * sentinels 0 (end of `next` chain) and -1 (no child) both become -1.
 *
 * Parity pinning: the reference cannot be compiled in this environment (no
 * Fortran compiler), and its own tests store no expected keys, permutations,
 * topologies or forces.  This restatement is therefore pinned only
 * statistically, against the force-error statistics the reference recorded in
 * benchmarks/forces_time_and_error/out/ (see tests/test_oracle.py).
 *
 * Floating point: compile with -ffp-contract=off.  Each Fortran operation is
 * then rounded separately, which is the semantics of the source text.  The one
 * place where the reference's own build (gfortran -O3 -march=native) may fuse a
 * multiply-add that changes an integer result is the sequential centre-of-mass
 * sum that feeds the key normalisation (morton_octree.f90:364-370); `fma_mode`
 * selects the separately-rounded (0) or the fused (1) form of that sum.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2
#define ORC_ECAPACITY 3
#define ORC_ELOST 4

static char g_err[256];
static int fail(int code, const char *msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}
const char *orc_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------- */
/* Shared helpers                                                             */
/* ------------------------------------------------------------------------- */

/* morton_octree.f90:279-301 (system_size_info), octree_default.f90:424-443
 * (node_size_center): centre of the bounding box and its largest extent. */
static void system_size_info(int64_t n, const double *x, const double *y, const double *z,
                             double info[4]) {
    double xmin = x[0], xmax = x[0], ymin = y[0], ymax = y[0], zmin = z[0], zmax = z[0];
    for (int64_t p = 1; p < n; ++p) {
        if (x[p] < xmin) xmin = x[p];
        if (x[p] > xmax) xmax = x[p];
        if (y[p] < ymin) ymin = y[p];
        if (y[p] > ymax) ymax = y[p];
        if (z[p] < zmin) zmin = z[p];
        if (z[p] > zmax) zmax = z[p];
    }
    info[0] = 0.5 * (xmin + xmax);
    info[1] = 0.5 * (ymin + ymax);
    info[2] = 0.5 * (zmin + zmax);
    double e = xmax - xmin;
    if (ymax - ymin > e) e = ymax - ymin;
    if (zmax - zmin > e) e = zmax - zmin;
    info[3] = e;
}

/* morton_octree.f90:184-213 (morton_key): quantise each axis to L bits and
 * interleave from the most significant bit down, octant digit (x<<2)+(y<<1)+z. */
static uint64_t morton_key(double x, double y, double z, int L) {
    int64_t scale = (int64_t)1 << L;
    int64_t ix = (int64_t)floor(x * (double)scale);
    int64_t iy = (int64_t)floor(y * (double)scale);
    int64_t iz = (int64_t)floor(z * (double)scale);
    if (ix > scale - 1) ix = scale - 1;
    if (iy > scale - 1) iy = scale - 1;
    if (iz > scale - 1) iz = scale - 1;
    uint64_t key = 0;
    for (int b = L - 1; b >= 0; --b) {
        uint64_t xb = ((uint64_t)ix >> b) & 1u;
        uint64_t yb = ((uint64_t)iy >> b) & 1u;
        uint64_t zb = ((uint64_t)iz >> b) & 1u;
        key = (key << 3) + ((xb << 2) + (yb << 1) + zb);
    }
    return key;
}

/* morton_octree.f90:519-560 (mergesort): top-down recursive merge sort of an
 * index array by key; ties take the left element, so the sort is stable. */
static void mergesort_rec(const uint64_t *keys, int32_t *perm, int32_t *tmp, int64_t left,
                          int64_t right) {
    if (left >= right) return;
    int64_t mid = (left + right) / 2;
    mergesort_rec(keys, perm, tmp, left, mid);
    mergesort_rec(keys, perm, tmp, mid + 1, right);
    int64_t i = left, j = mid + 1, k = left;
    while (i <= mid && j <= right) {
        if (keys[perm[i]] <= keys[perm[j]]) tmp[k++] = perm[i++];
        else tmp[k++] = perm[j++];
    }
    while (i <= mid) tmp[k++] = perm[i++];
    while (j <= right) tmp[k++] = perm[j++];
    memcpy(perm + left, tmp + left, (size_t)(right - left + 1) * sizeof(int32_t));
}

/* morton_octree.f90:501-517 (argsort). The Fortran recursion splits at
 * (left+right)/2 on 1-based bounds; a stable sort's output does not depend on
 * the split, so the 0-based split here yields the same permutation. */
int orc_argsort(int64_t n, const uint64_t *keys, int32_t *perm) {
    if (n <= 0) return fail(ORC_EINVAL, "argsort: n must be positive");
    int32_t *tmp = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    if (!tmp) return fail(ORC_ENOMEM, "argsort: out of memory");
    for (int64_t i = 0; i < n; ++i) perm[i] = (int32_t)i;
    mergesort_rec(keys, perm, tmp, 0, n - 1);
    free(tmp);
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Morton octree (fortran/morton/morton_octree.f90)                           */
/* ------------------------------------------------------------------------- */

/* Steps 1-5 of generate_nodes, morton_octree.f90:359-395: bounding box, the
 * sequential FP64 centre of mass, normalisation into [0,1]^3 recentred at 1/2,
 * and the keys (or choose_depth when L == 0).  keys[] is in ORIGINAL order.
 * out_com4 = (qcm_x, qcm_y, qcm_z, total mass); out_ssa = 1.2*extent. */
int orc_morton_keys(int64_t n, const double *m, const double *x, const double *y,
                    const double *z, int L, double ssa_amp, int fma_mode, uint64_t *keys,
                    int *out_L, double *out_com4, double *out_ssa) {
    if (n <= 0) return fail(ORC_EINVAL, "keys: n must be positive");
    if (L < 0 || L > 21) return fail(ORC_EINVAL, "keys: depth must be in 0..21");
    double ssi[4];
    system_size_info(n, x, y, z, ssi);                      /* :360 */
    double ssa = ssa_amp * ssi[3];                          /* :361 */
    double qcm[3] = {0.0, 0.0, 0.0}, mass = 0.0;            /* :364-370 */
    for (int64_t p = 0; p < n; ++p) {
        if (fma_mode) {
            qcm[0] = fma(m[p], x[p], qcm[0]);
            qcm[1] = fma(m[p], y[p], qcm[1]);
            qcm[2] = fma(m[p], z[p], qcm[2]);
        } else {
            qcm[0] = qcm[0] + m[p] * x[p];
            qcm[1] = qcm[1] + m[p] * y[p];
            qcm[2] = qcm[2] + m[p] * z[p];
        }
        mass = mass + m[p];
    }
    qcm[0] = qcm[0] / mass;
    qcm[1] = qcm[1] / mass;
    qcm[2] = qcm[2] / mass;
    double *vx = (double *)malloc((size_t)n * 3 * sizeof(double));
    if (!vx) return fail(ORC_ENOMEM, "keys: out of memory");
    double *vy = vx + n, *vz = vy + n;
    for (int64_t p = 0; p < n; ++p) {                       /* :373-376 */
        vx[p] = x[p] - qcm[0];
        vy[p] = y[p] - qcm[1];
        vz[p] = z[p] - qcm[2];
    }
    for (int64_t p = 0; p < n; ++p) {
        vx[p] = vx[p] / ssa;
        vy[p] = vy[p] / ssa;
        vz[p] = vz[p] / ssa;
    }
    system_size_info(n, vx, vy, vz, ssi);                   /* :380 */
    for (int64_t p = 0; p < n; ++p) {                       /* :382-384 */
        vx[p] = vx[p] + 0.5 - ssi[0];
        vy[p] = vy[p] + 0.5 - ssi[1];
        vz[p] = vz[p] + 0.5 - ssi[2];
    }
    if (L == 0) {
        /* choose_depth, morton_octree.f90:217-244: smallest L with unique keys,
         * by brute force (O(N^2) per level, as in the reference). */
        L = 1;
        for (;;) {
            int unique = 1;
            for (int64_t p = 0; p < n && unique; ++p) {
                keys[p] = morton_key(vx[p], vy[p], vz[p], L);
                for (int64_t q = 0; q < p; ++q)
                    if (keys[q] == keys[p]) { unique = 0; break; }
            }
            if (unique) break;
            if (++L > 21) {
                free(vx);
                return fail(ORC_EINVAL, "choose_depth: keys never become unique (coincident bodies)");
            }
        }
    } else {
        for (int64_t p = 0; p < n; ++p) keys[p] = morton_key(vx[p], vy[p], vz[p], L);
    }
    free(vx);
    if (out_L) *out_L = L;
    if (out_com4) {
        out_com4[0] = qcm[0]; out_com4[1] = qcm[1]; out_com4[2] = qcm[2]; out_com4[3] = mass;
    }
    if (out_ssa) *out_ssa = ssa;
    return ORC_OK;
}

typedef struct {
    int64_t n;
    int L;
    double ssa;
    double com[3], mass;
    int use_quad;
    int32_t *perm;      /* sorted position -> original index */
    uint64_t *skeys;    /* keys in sorted order */
    double *ms, *qx, *qy, *qz; /* masses and positions in sorted order */
    int64_t nnodes, cap;
    int64_t *level_begin, *level_end; /* L+1 entries each, node index ranges */
    int64_t *prefix;
    int32_t *level, *first, *last, *parent, *nchild, *child, *next;
    double *size2, *nmass, *qcm, *quad;
    double *oct;        /* 14 per node, only after orc_morton_octupoles */
} orc_morton;

void orc_morton_free(orc_morton *t) {
    if (!t) return;
    free(t->perm); free(t->skeys); free(t->ms);
    free(t->level_begin); free(t->level_end);
    free(t->prefix); free(t->level); free(t->first); free(t->last); free(t->parent);
    free(t->nchild); free(t->child); free(t->next);
    free(t->size2); free(t->nmass); free(t->qcm); free(t->quad); free(t->oct);
    free(t);
}

/* morton_octree.f90:257-275 (create_node). */
static void create_node(orc_morton *t, int64_t idx, int level, int64_t pref, int64_t first,
                        int64_t last, double mass, const double qcm[3], double size) {
    t->level[idx] = level;
    t->prefix[idx] = pref;
    t->first[idx] = (int32_t)first;
    t->last[idx] = (int32_t)last;
    t->nmass[idx] = mass;
    t->qcm[3 * idx + 0] = qcm[0];
    t->qcm[3 * idx + 1] = qcm[1];
    t->qcm[3 * idx + 2] = qcm[2];
    t->size2[idx] = size * size;
    t->parent[idx] = -1;
    t->nchild[idx] = 0;
    for (int c = 0; c < 8; ++c) t->child[8 * idx + c] = -1;
    for (int c = 0; c < 6; ++c) t->quad[6 * idx + c] = 0.0;
}

/* morton_octree.f90:304-326 (build_next): threaded depth-first successor. */
static void build_next(orc_morton *t, int64_t idx, int64_t sibling) {
    t->next[idx] = (int32_t)sibling;
    int nc = t->nchild[idx];
    if (nc == 0) return;
    for (int i = 0; i < nc - 1; ++i) build_next(t, t->child[8 * idx + i], t->child[8 * idx + i + 1]);
    build_next(t, t->child[8 * idx + nc - 1], sibling);
}

/* morton_octree.f90:562-625 (evaluate_quadrupoles): bottom-up by level; nodes
 * with <= 1 child sum their particles directly about the node centre of mass,
 * the others translate their children's moments (parallel-axis rule). */
static void evaluate_quadrupoles(orc_morton *t) {
    for (int level = t->L; level >= 0; --level) {
        for (int64_t node = t->level_begin[level]; node <= t->level_end[level]; ++node) {
            double *q = t->quad + 6 * node;
            const double *c = t->qcm + 3 * node;
            for (int k = 0; k < 6; ++k) q[k] = 0.0;
            if (t->nchild[node] <= 1) {
                for (int64_t p = t->first[node]; p <= t->last[node]; ++p) {
                    double pm = t->ms[p];
                    double dxi = t->qx[p] - c[0];
                    double dyi = t->qy[p] - c[1];
                    double dzi = t->qz[p] - c[2];
                    q[0] = q[0] + pm * (dxi * dxi);
                    q[1] = q[1] + pm * (dyi * dyi);
                    q[2] = q[2] + pm * (dzi * dzi);
                    q[3] = q[3] + pm * dxi * dyi;
                    q[4] = q[4] + pm * dxi * dzi;
                    q[5] = q[5] + pm * dyi * dzi;
                }
            } else {
                for (int cp = 0; cp < t->nchild[node]; ++cp) {
                    int64_t ch = t->child[8 * node + cp];
                    const double *qc = t->quad + 6 * ch;
                    double pm = t->nmass[ch];
                    double dxi = t->qcm[3 * ch + 0] - c[0];
                    double dyi = t->qcm[3 * ch + 1] - c[1];
                    double dzi = t->qcm[3 * ch + 2] - c[2];
                    q[0] = q[0] + qc[0] + pm * dxi * dxi;
                    q[1] = q[1] + qc[1] + pm * dyi * dyi;
                    q[2] = q[2] + qc[2] + pm * dzi * dzi;
                    q[3] = q[3] + qc[3] + pm * dxi * dyi;
                    q[4] = q[4] + qc[4] + pm * dxi * dzi;
                    q[5] = q[5] + qc[5] + pm * dyi * dzi;
                }
            }
        }
    }
}

/* morton_octree.f90:73-111 (init) and :328-499 (generate_nodes). */
int orc_morton_build(int64_t n, const double *m, const double *x, const double *y,
                     const double *z, int L, double ssa_amp, int fma_mode, int use_quad,
                     orc_morton **out) {
    *out = NULL;
    if (n <= 0 || n > 0x7fffffff) return fail(ORC_EINVAL, "morton: n out of range");
    orc_morton *t = (orc_morton *)calloc(1, sizeof(orc_morton));
    if (!t) return fail(ORC_ENOMEM, "morton: out of memory");
    t->n = n;
    t->use_quad = use_quad;
    uint64_t *keys = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    if (!keys) { orc_morton_free(t); return fail(ORC_ENOMEM, "morton: out of memory"); }
    double com4[4];
    int rc = orc_morton_keys(n, m, x, y, z, L, ssa_amp, fma_mode, keys, &t->L, com4, &t->ssa);
    if (rc) { free(keys); orc_morton_free(t); return rc; }
    L = t->L;
    t->com[0] = com4[0]; t->com[1] = com4[1]; t->com[2] = com4[2]; t->mass = com4[3];

    t->perm = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    t->skeys = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    t->ms = (double *)malloc((size_t)n * 4 * sizeof(double));
    if (!t->perm || !t->skeys || !t->ms) { free(keys); orc_morton_free(t); return fail(ORC_ENOMEM, "morton: out of memory"); }
    t->qx = t->ms + n; t->qy = t->qx + n; t->qz = t->qy + n;
    rc = orc_argsort(n, keys, t->perm);                       /* :404 */
    if (rc) { free(keys); orc_morton_free(t); return rc; }
    for (int64_t p = 0; p < n; ++p) {                         /* :408-417 */
        int32_t o = t->perm[p];
        t->skeys[p] = keys[o];
        t->ms[p] = m[o]; t->qx[p] = x[o]; t->qy[p] = y[o]; t->qz[p] = z[o];
    }
    free(keys);

    int64_t cap = (int64_t)(L + 1) * n;                       /* :421 */
    t->cap = cap;
    t->level_begin = (int64_t *)malloc((size_t)(L + 1) * sizeof(int64_t));
    t->level_end = (int64_t *)malloc((size_t)(L + 1) * sizeof(int64_t));
    t->prefix = (int64_t *)malloc((size_t)cap * sizeof(int64_t));
    t->level = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    t->first = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    t->last = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    t->parent = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    t->nchild = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    t->next = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    t->child = (int32_t *)malloc((size_t)cap * 8 * sizeof(int32_t));
    t->size2 = (double *)malloc((size_t)cap * sizeof(double));
    t->nmass = (double *)malloc((size_t)cap * sizeof(double));
    t->qcm = (double *)malloc((size_t)cap * 3 * sizeof(double));
    t->quad = (double *)malloc((size_t)cap * 6 * sizeof(double));
    if (!t->level_begin || !t->level_end || !t->prefix || !t->level || !t->first || !t->last ||
        !t->parent || !t->nchild || !t->next || !t->child || !t->size2 || !t->nmass || !t->qcm ||
        !t->quad) {
        orc_morton_free(t);
        return fail(ORC_ENOMEM, "morton: out of memory for nodes");
    }

    /* root, :424-427 */
    int64_t nnodes = 0;
    create_node(t, 0, 0, (int64_t)(t->skeys[0] >> (3 * L)), 0, n - 1, t->mass, t->com, t->ssa);
    nnodes = 1;
    t->level_begin[0] = 0;
    t->level_end[0] = 0;
    /* level loop, :430-493 */
    for (int level = 1; level <= L; ++level) {
        t->level_begin[level] = nnodes;
        double size = t->ssa * ldexp(1.0, -level);
        int shift = 3 * (L - level);
        for (int64_t par = t->level_begin[level - 1]; par <= t->level_end[level - 1]; ++par) {
            int64_t first = t->first[par], last = t->last[par];
            int64_t current = -1, child_first = 0;
            double mass = 0.0, qcm[3] = {0.0, 0.0, 0.0};
            for (int64_t i = first; i <= last; ++i) {
                int64_t pref = (int64_t)(t->skeys[i] >> shift);
                if (current == -1) {
                    current = pref;
                    child_first = i;
                    mass = t->ms[i];
                    qcm[0] = mass * t->qx[i]; qcm[1] = mass * t->qy[i]; qcm[2] = mass * t->qz[i];
                } else if (pref != current) {
                    qcm[0] = qcm[0] / mass; qcm[1] = qcm[1] / mass; qcm[2] = qcm[2] / mass;
                    create_node(t, nnodes, level, current, child_first, i - 1, mass, qcm, size);
                    t->parent[nnodes] = (int32_t)par;
                    t->child[8 * par + t->nchild[par]] = (int32_t)nnodes;
                    t->nchild[par] += 1;
                    nnodes += 1;
                    current = pref;
                    child_first = i;
                    mass = t->ms[i];
                    qcm[0] = mass * t->qx[i]; qcm[1] = mass * t->qy[i]; qcm[2] = mass * t->qz[i];
                } else {
                    mass = mass + t->ms[i];
                    qcm[0] = qcm[0] + t->ms[i] * t->qx[i];
                    qcm[1] = qcm[1] + t->ms[i] * t->qy[i];
                    qcm[2] = qcm[2] + t->ms[i] * t->qz[i];
                }
            }
            qcm[0] = qcm[0] / mass; qcm[1] = qcm[1] / mass; qcm[2] = qcm[2] / mass;
            create_node(t, nnodes, level, current, child_first, last, mass, qcm, size);
            t->parent[nnodes] = (int32_t)par;
            t->child[8 * par + t->nchild[par]] = (int32_t)nnodes;
            t->nchild[par] += 1;
            nnodes += 1;
        }
        t->level_end[level] = nnodes - 1;
    }
    t->nnodes = nnodes;
    build_next(t, 0, -1);                                     /* :498 */
    if (use_quad) evaluate_quadrupoles(t);                    /* :105-110 */
    *out = t;
    return ORC_OK;
}

int orc_morton_info(const orc_morton *t, int64_t *nnodes, int *L, double *ssa, double *com4) {
    if (nnodes) *nnodes = t->nnodes;
    if (L) *L = t->L;
    if (ssa) *ssa = t->ssa;
    if (com4) { com4[0] = t->com[0]; com4[1] = t->com[1]; com4[2] = t->com[2]; com4[3] = t->mass; }
    return ORC_OK;
}

int orc_morton_get_sorted(const orc_morton *t, uint64_t *keys, int32_t *perm) {
    if (keys) memcpy(keys, t->skeys, (size_t)t->n * sizeof(uint64_t));
    if (perm) memcpy(perm, t->perm, (size_t)t->n * sizeof(int32_t));
    return ORC_OK;
}

int orc_morton_get_levels(const orc_morton *t, int64_t *level_begin, int64_t *level_end) {
    memcpy(level_begin, t->level_begin, (size_t)(t->L + 1) * sizeof(int64_t));
    memcpy(level_end, t->level_end, (size_t)(t->L + 1) * sizeof(int64_t));
    return ORC_OK;
}

/* Copies the node arrays (any pointer may be NULL). child8 is nnodes x 8,
 * qcm3 nnodes x 3, quad6 nnodes x 6, all row-major. */
int orc_morton_get_nodes(const orc_morton *t, int64_t *prefix, int32_t *level, double *size2,
                         int32_t *first, int32_t *last, int32_t *parent, int32_t *nchild,
                         int32_t *child8, int32_t *next, double *mass, double *qcm3,
                         double *quad6) {
    size_t nn = (size_t)t->nnodes;
    if (prefix) memcpy(prefix, t->prefix, nn * sizeof(int64_t));
    if (level) memcpy(level, t->level, nn * sizeof(int32_t));
    if (size2) memcpy(size2, t->size2, nn * sizeof(double));
    if (first) memcpy(first, t->first, nn * sizeof(int32_t));
    if (last) memcpy(last, t->last, nn * sizeof(int32_t));
    if (parent) memcpy(parent, t->parent, nn * sizeof(int32_t));
    if (nchild) memcpy(nchild, t->nchild, nn * sizeof(int32_t));
    if (child8) memcpy(child8, t->child, nn * 8 * sizeof(int32_t));
    if (next) memcpy(next, t->next, nn * sizeof(int32_t));
    if (mass) memcpy(mass, t->nmass, nn * sizeof(double));
    if (qcm3) memcpy(qcm3, t->qcm, nn * 3 * sizeof(double));
    if (quad6) memcpy(quad6, t->quad, nn * 6 * sizeof(double));
    return ORC_OK;
}

/* The octupole part of a cell's field, octree_default.f90:1012-1063 (the
 * insertion tree's bh_forces_over_p), on the raw third moments o[14] of the
 * node about its centre of mass: the same expression as octree_walk below.
 * invR, invR2 and invR5 are of the softened distance. */
static void octupole_terms(const double *o, double dx, double dy, double dz, double invR,
                           double invR2, double invR5, double O[3]) {
    (void)invR2;
    double invR7 = invR5 * invR * invR;
    double invR9 = invR7 * invR * invR;
    double Ox = -1.5 * invR5 * o[11];
    double Oy = -1.5 * invR5 * o[12];
    double Oz = -1.5 * invR5 * o[13];
    double Oc = 7.5 * invR7 * (dx * o[11] + dy * o[12] + dz * o[13]);
    Ox = Ox + dx * Oc; Oy = Oy + dy * Oc; Oz = Oz + dz * Oc;
    double ddx = dx * dx, ddy = dy * dy, ddz = dz * dz;
    Ox = Ox + 7.5 * invR7 * (ddx * o[0] + ddy * o[1] + ddz * o[2] + 2.0 * dx * dy * o[3] +
                             2.0 * dx * dz * o[6] + 2.0 * dy * dz * o[9]);
    Oy = Oy + 7.5 * invR7 * (ddx * o[3] + ddy * o[4] + ddz * o[5] + 2.0 * dx * dy * o[1] +
                             2.0 * dx * dz * o[9] + 2.0 * dy * dz * o[7]);
    Oz = Oz + 7.5 * invR7 * (ddx * o[6] + ddy * o[7] + ddz * o[8] + 2.0 * dx * dy * o[9] +
                             2.0 * dx * dz * o[2] + 2.0 * dy * dz * o[5]);
    Oc = -17.5 * invR9 *
         (ddx * dx * o[0] + ddy * dy * o[4] + ddz * dz * o[8] + 3.0 * ddx * dy * o[3] +
          3.0 * ddx * dz * o[6] + 3.0 * ddy * dx * o[1] + 3.0 * ddy * dz * o[7] +
          3.0 * ddz * dx * o[2] + 3.0 * ddz * dy * o[5] + 6.0 * dx * dy * dz * o[9]);
    O[0] = Ox + dx * Oc; O[1] = Oy + dy * Oc; O[2] = Oz + dz * Oc;
}

/* morton_octree.f90:627-766 (barnes_hut): stackless walk over `next` links for
 * sorted particle p.  Returns the force (G m_p a_p).  cnt[0] counts body-body
 * interactions (leaf particles and single-particle nodes), cnt[1] counts
 * multipole (quadrupole) cell interactions.  mult 0 monopole, 1 quadrupole
 * (the reference's two options); mult 8 adds the octupole terms of the
 * insertion tree's walk to the quadrupole (needs orc_morton_octupoles). */
static void morton_walk(const orc_morton *t, int64_t p, double theta2, double G, double eps2,
                        int mult, double f[3], int64_t cnt[2]) {
    double mp = t->ms[p];
    double qp0 = t->qx[p], qp1 = t->qy[p], qp2 = t->qz[p];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    int64_t npp = 0, npc = 0;
    int64_t idx = 0;
    while (idx != -1) {
        int only_one = (t->first[idx] == t->last[idx]);
        /* :666 compares `last` with the Fortran index 0, which no particle has,
         * so the branch never fires; restated with the 0-based equivalent -1. */
        if (only_one && t->last[idx] == -1) { idx = t->next[idx]; continue; }
        if (t->nchild[idx] == 0) {                               /* :672-691 */
            for (int64_t b = t->first[idx]; b <= t->last[idx]; ++b) {
                if (p == b) continue;
                double dx = t->qx[b] - qp0, dy = t->qy[b] - qp1, dz = t->qz[b] - qp2;
                double dist2 = dx * dx + dy * dy + dz * dz + eps2;
                double invdist3 = 1.0 / sqrt(dist2);
                invdist3 = invdist3 * invdist3 * invdist3;
                double ff = G * mp * t->ms[b] * invdist3;
                fx = fx + ff * dx; fy = fy + ff * dy; fz = fz + ff * dz;
                npp++;
            }
            idx = t->next[idx];
            continue;
        }
        if (t->first[idx] <= p && p <= t->last[idx]) {           /* :694-697 */
            idx = t->child[8 * idx];
            continue;
        }
        const double *c = t->qcm + 3 * idx;                      /* :701-704 */
        double dx = c[0] - qp0, dy = c[1] - qp1, dz = c[2] - qp2;
        double dist2 = dx * dx + dy * dy + dz * dz;
        if (only_one || t->size2[idx] <= theta2 * dist2) {       /* :706 */
            if (t->nmass[idx] > 0) {
                dist2 = dist2 + eps2;
                if (!mult || only_one) {                         /* :711-718 */
                    double invdist3 = 1.0 / sqrt(dist2);
                    invdist3 = invdist3 * invdist3 * invdist3;
                    double ff = G * mp * t->nmass[idx] * invdist3;
                    fx = fx + ff * dx; fy = fy + ff * dy; fz = fz + ff * dz;
                    if (only_one) npp++; else npc++;
                } else {                                         /* :721-753 */
                    const double *q = t->quad + 6 * idx;
                    double invR = 1.0 / sqrt(dist2);
                    double invR2 = 1.0 / dist2;
                    double invR3 = invR * invR2;
                    double invR5 = invR3 * invR * invR;
                    double mx = dx * invR3 * t->nmass[idx];
                    double my = dy * invR3 * t->nmass[idx];
                    double mz = dz * invR3 * t->nmass[idx];
                    double mxi2 = q[0], myi2 = q[1], mzi2 = q[2], mxyi = q[3], mxzi = q[4], myzi = q[5];
                    double dx2 = 15.0 * dx * dx * invR2 - 3.0;
                    double dy2 = 15.0 * dy * dy * invR2 - 3.0;
                    double dz2 = 15.0 * dz * dz * invR2 - 3.0;
                    double dxyz = 15.0 * dx * dy * dz * invR2;
                    double Qx = (mxi2 * (dx2 - 6.0) + myi2 * dy2 + mzi2 * dz2) * 0.5 * dx;
                    double Qy = (myi2 * (dy2 - 6.0) + mzi2 * dz2 + mxi2 * dx2) * 0.5 * dy;
                    double Qz = (mzi2 * (dz2 - 6.0) + mxi2 * dx2 + myi2 * dy2) * 0.5 * dz;
                    Qx = Qx + mxyi * dy * dx2 + mxzi * dz * dx2 + myzi * dxyz;
                    Qy = Qy + myzi * dz * dy2 + mxyi * dx * dy2 + mxzi * dxyz;
                    Qz = Qz + mxzi * dx * dz2 + myzi * dy * dz2 + mxyi * dxyz;
                    double O[3] = {0.0, 0.0, 0.0};
                    if (mult == 8) octupole_terms(t->oct + 14 * idx, dx, dy, dz, invR, invR2, invR5, O);
                    fx = fx + G * mp * (mx + invR5 * Qx + O[0]);
                    fy = fy + G * mp * (my + invR5 * Qy + O[1]);
                    fz = fz + G * mp * (mz + invR5 * Qz + O[2]);
                    npc++;
                }
            }
            idx = t->next[idx];
            continue;
        }
        idx = t->child[8 * idx];                                 /* :761-763 */
    }
    f[0] = fx; f[1] = fy; f[2] = fz;
    if (cnt) { cnt[0] = npp; cnt[1] = npc; }
}

static void direct_moments(const orc_morton *t, int64_t first, int64_t last, const double c[3],
                           double *Q, double *O);

/* Raw third moments of every node about its centre of mass, summed directly
 * over the node's particles with the summary sums of octree_default.f90
 * :875-880 (the Morton module itself stops at the quadrupole).  Lets the walk
 * above run with mult 8: the Morton tree's topology with the octupole terms
 * of octree_default.f90:1012-1063. */
int orc_morton_octupoles(orc_morton *t) {
    if (t->oct) return ORC_OK;
    t->oct = (double *)malloc((size_t)t->nnodes * 14 * sizeof(double));
    if (!t->oct) return fail(ORC_ENOMEM, "octupoles: out of memory");
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (int64_t j = 0; j < t->nnodes; ++j) {
        double Q[6];
        if (t->first[j] < 0) { for (int k = 0; k < 14; ++k) t->oct[14 * j + k] = 0.0; continue; }
        direct_moments(t, t->first[j], t->last[j], t->qcm + 3 * j, Q, t->oct + 14 * j);
    }
    return ORC_OK;
}

/* morton_octree.f90:150-180 (forces_par): forces for every particle, written
 * back through the permutation into ORIGINAL order.  out is SoA: fx[n], fy[n],
 * fz[n] (the memory layout of the api3d (N,3) Fortran result). */
int orc_morton_forces(const orc_morton *t, double G, double eps2, double theta2, int mult,
                      double *out, int nthreads) {
    int64_t n = t->n;
    if (mult == 8 && !t->oct) return fail(ORC_EINVAL, "forces: mult 8 needs orc_morton_octupoles");
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int64_t p = 0; p < n; ++p) {
        double f[3];
        morton_walk(t, p, theta2, G, eps2, mult, f, NULL);
        int64_t o = t->perm[p];
        out[o] = f[0]; out[n + o] = f[1]; out[2 * n + o] = f[2];
    }
    (void)nthreads;
    return ORC_OK;
}

/* Forces on a subset of targets given by ORIGINAL index.  out is SoA over the
 * targets; counts (optional) receives 2 per target: body-body and cell terms. */
int orc_morton_forces_targets(const orc_morton *t, double G, double eps2, double theta2, int mult,
                              int64_t nt, const int64_t *targets, double *out, int64_t *counts,
                              int nthreads) {
    int64_t n = t->n;
    if (mult == 8 && !t->oct) return fail(ORC_EINVAL, "targets: mult 8 needs orc_morton_octupoles");
    int32_t *inv = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    if (!inv) return fail(ORC_ENOMEM, "targets: out of memory");
    for (int64_t p = 0; p < n; ++p) inv[t->perm[p]] = (int32_t)p;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
    for (int64_t k = 0; k < nt; ++k) {
        double f[3];
        int64_t c[2];
        morton_walk(t, inv[targets[k]], theta2, G, eps2, mult, f, c);
        out[k] = f[0]; out[nt + k] = f[1]; out[2 * nt + k] = f[2];
        if (counts) { counts[2 * k] = c[0]; counts[2 * k + 1] = c[1]; }
    }
    (void)nthreads;
    free(inv);
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Insertion octree (fortran/octree_default.f90)                              */
/* ------------------------------------------------------------------------- */

typedef struct {
    int64_t n;
    int method, multipole, group_size, max_depth, most_depth;
    double side_amp;
    double *m, *x, *y, *z;
    int64_t nnodes, cap;
    double *cx, *cy, *cz, *halfside, *L2, *mass, *qx, *qy, *qz, *quad, *oct;
    int32_t *particle, *type, *child, *depth;
    /* grouped BH */
    int32_t *count, *first, *last, *order, *groups;
    int64_t ngroups;
    double *gx, *gy, *gz, *gm;
    int err;
} orc_octree;

void orc_octree_free(orc_octree *t) {
    if (!t) return;
    free(t->m); free(t->cx); free(t->quad); free(t->oct);
    free(t->particle); free(t->type); free(t->child); free(t->depth);
    /* first, last and groups live inside the `count` allocation */
    free(t->count); free(t->order); free(t->gx);
    free(t);
}

/* octree_default.f90:178-282 (pre_init).  method: 10/11/12 classic BH with
 * monopole/quadrupole/octupole, 20/21/22 Dehnen's dual-tree method, 30/31/32
 * grouped BH.  max_nodes == 0 keeps the
 * reference's node budget (3N for N >= 1000, else 10N, :219-223); a larger
 * budget may be passed for strongly clustered inputs where the reference would
 * stop with "INSUFFICIENT NUMBER OF NODES". */
int orc_octree_create(int64_t n, const double *m, int method, int group_size, int64_t max_nodes,
                      orc_octree **out) {
    *out = NULL;
    if (n <= 0 || n > 0x3fffffff) return fail(ORC_EINVAL, "octree: n out of range");
    int mp;
    switch (method) {
    case 10: case 30: mp = 1; break;
    case 11: case 31: mp = 4; break;
    case 12: case 32: mp = 8; break;
    case 20: mp = 1; break;
    case 21: mp = 4; break;
    case 22: mp = 8; break;
    default: return fail(ORC_EINVAL, "octree: method must be 10-12, 20-22 or 30-32");
    }
    orc_octree *t = (orc_octree *)calloc(1, sizeof(orc_octree));
    if (!t) return fail(ORC_ENOMEM, "octree: out of memory");
    t->n = n; t->method = method; t->multipole = mp;
    t->group_size = group_size > 0 ? group_size : 64;
    t->max_depth = 25; t->side_amp = 1.2;
    t->cap = max_nodes > 0 ? max_nodes : (n >= 1000 ? 3 * n : 10 * n);
    int64_t c = t->cap;
    t->m = (double *)malloc((size_t)n * 4 * sizeof(double));
    t->cx = (double *)malloc((size_t)c * 10 * sizeof(double));
    t->quad = (double *)calloc((size_t)c * 6, sizeof(double));
    t->oct = (double *)calloc((size_t)c * 14, sizeof(double));
    t->particle = (int32_t *)malloc((size_t)c * sizeof(int32_t));
    t->type = (int32_t *)malloc((size_t)c * sizeof(int32_t));
    t->child = (int32_t *)malloc((size_t)c * 8 * sizeof(int32_t));
    t->depth = (int32_t *)malloc((size_t)c * sizeof(int32_t));
    if (!t->m || !t->cx || !t->quad || !t->oct || !t->particle || !t->type || !t->child || !t->depth) {
        orc_octree_free(t);
        return fail(ORC_ENOMEM, "octree: out of memory for nodes");
    }
    t->x = t->m + n; t->y = t->x + n; t->z = t->y + n;
    t->cy = t->cx + c; t->cz = t->cy + c; t->halfside = t->cz + c; t->L2 = t->halfside + c;
    t->mass = t->L2 + c; t->qx = t->mass + c; t->qy = t->qx + c; t->qz = t->qy + c;
    memcpy(t->m, m, (size_t)n * sizeof(double));
    *out = t;
    return ORC_OK;
}

/* octree_default.f90:445-479 (add_node). */
static int64_t add_node(orc_octree *t, double cx, double cy, double cz, double side, int depth) {
    int64_t idx = t->nnodes++;
    if (idx >= t->cap) { t->err = ORC_ECAPACITY; t->nnodes = t->cap; return -1; }
    for (int k = 0; k < 8; ++k) t->child[8 * idx + k] = -1;
    t->type[idx] = 1;
    t->depth[idx] = depth;
    if (depth > t->most_depth) t->most_depth = depth;
    t->cx[idx] = cx; t->cy[idx] = cy; t->cz[idx] = cz;
    t->halfside[idx] = side / 2.0;
    t->L2[idx] = side * side;
    t->mass[idx] = 0.0; t->qx[idx] = 0.0; t->qy[idx] = 0.0; t->qz[idx] = 0.0;
    t->particle[idx] = -1;
    return idx;
}

static void add(orc_octree *t, int64_t node, int64_t p);

/* octree_default.f90:515-545 (add_to_subnode) with :481-513 (allocate_subnode). */
static void add_to_subnode(orc_octree *t, int64_t node, int64_t p) {
    if (t->err) return;
    int ix = t->x[p] >= t->cx[node];
    int iy = t->y[p] < t->cy[node];
    int iz = t->z[p] < t->cz[node];
    int index = ix + 2 * iy + 4 * iz; /* Fortran subnode_index - 1 */
    int64_t sub = t->child[8 * node + index];
    if (sub == -1) {
        double h = t->halfside[node];
        double h_half = h / 2.0;
        int sx = (index & 1) ? 1 : -1;
        int sy = (index & 2) ? -1 : 1;
        int sz = (index & 4) ? -1 : 1;
        sub = add_node(t, t->cx[node] + sx * h_half, t->cy[node] + sy * h_half,
                       t->cz[node] + sz * h_half, h, t->depth[node] + 1);
        if (sub < 0) return;
        t->child[8 * node + index] = (int32_t)sub;
    }
    add(t, sub, p);
}

/* octree_default.f90:547-580 (add). */
static void add(orc_octree *t, int64_t node, int64_t p) {
    if (t->err) return;
    if (t->particle[node] == -1 && t->type[node] == 1) { t->particle[node] = (int32_t)p; return; }
    if (t->type[node] == 1) {
        t->type[node] = 2;
        int64_t old_p = t->particle[node];
        t->particle[node] = -1;
        if (t->depth[node] < t->max_depth) add_to_subnode(t, node, old_p);
    }
    if (t->depth[node] < t->max_depth) add_to_subnode(t, node, p);
}

/* octree_default.f90:582-628 (incorporate_particles): monopole upward pass. */
static void incorporate_particles(orc_octree *t) {
    for (int64_t node = t->nnodes - 1; node >= 0; --node) {
        if (t->type[node] == 1) {
            int64_t p = t->particle[node];
            if (p == -1) continue;
            t->mass[node] = t->m[p]; t->qx[node] = t->x[p]; t->qy[node] = t->y[p]; t->qz[node] = t->z[p];
        } else {
            t->mass[node] = 0.0; t->qx[node] = 0.0; t->qy[node] = 0.0; t->qz[node] = 0.0;
            for (int c = 0; c < 8; ++c) {
                int64_t ch = t->child[8 * node + c];
                if (ch == -1) continue;
                t->mass[node] = t->mass[node] + t->mass[ch];
                t->qx[node] = t->qx[node] + t->mass[ch] * t->qx[ch];
                t->qy[node] = t->qy[node] + t->mass[ch] * t->qy[ch];
                t->qz[node] = t->qz[node] + t->mass[ch] * t->qz[ch];
            }
            t->qx[node] = t->qx[node] / t->mass[node];
            t->qy[node] = t->qy[node] / t->mass[node];
            t->qz[node] = t->qz[node] / t->mass[node];
        }
    }
}

/* octree_default.f90:744-882 (evaluate_multipole): mass/COM, quadrupole via the
 * parallel-axis rule and octupole raw third moments with the 3 d Q cross
 * terms, plus the summary sums oct(11..14). */
static void evaluate_multipole(orc_octree *t) {
    int oct = t->multipole > 4;
    for (int64_t node = t->nnodes - 1; node >= 0; --node) {
        if (t->type[node] == 1) {
            int64_t p = t->particle[node];
            if (p == -1) continue;
            t->mass[node] = t->m[p]; t->qx[node] = t->x[p]; t->qy[node] = t->y[p]; t->qz[node] = t->z[p];
            continue;
        }
        if (t->depth[node] == t->max_depth) continue;
        t->mass[node] = 0.0; t->qx[node] = 0.0; t->qy[node] = 0.0; t->qz[node] = 0.0;
        for (int c = 0; c < 8; ++c) {
            int64_t d = t->child[8 * node + c];
            if (d == -1) continue;
            t->mass[node] = t->mass[node] + t->mass[d];
            t->qx[node] = t->qx[node] + t->mass[d] * t->qx[d];
            t->qy[node] = t->qy[node] + t->mass[d] * t->qy[d];
            t->qz[node] = t->qz[node] + t->mass[d] * t->qz[d];
        }
        t->qx[node] = t->qx[node] / t->mass[node];
        t->qy[node] = t->qy[node] / t->mass[node];
        t->qz[node] = t->qz[node] / t->mass[node];
        double *Q = t->quad + 6 * node, *O = t->oct + 14 * node;
        for (int c = 0; c < 8; ++c) {
            int64_t d = t->child[8 * node + c];
            if (d == -1) continue;
            double pm = t->mass[d];
            double dxi = t->qx[d] - t->qx[node];
            double dyi = t->qy[d] - t->qy[node];
            double dzi = t->qz[d] - t->qz[node];
            const double *Qd = t->quad + 6 * d, *Od = t->oct + 14 * d;
            if (t->type[d] == 2) {
                for (int k = 0; k < 6; ++k) Q[k] = Q[k] + Qd[k];
                if (oct) for (int k = 0; k < 14; ++k) O[k] = O[k] + Od[k];
            }
            Q[0] = Q[0] + pm * (dxi * dxi);
            Q[1] = Q[1] + pm * (dyi * dyi);
            Q[2] = Q[2] + pm * (dzi * dzi);
            Q[3] = Q[3] + pm * dxi * dyi;
            Q[4] = Q[4] + pm * dxi * dzi;
            Q[5] = Q[5] + pm * dyi * dzi;
            if (oct) {
                O[0] = O[0] + pm * dxi * (dxi * dxi);
                O[1] = O[1] + pm * dxi * (dyi * dyi);
                O[2] = O[2] + pm * dxi * (dzi * dzi);
                O[3] = O[3] + pm * dyi * (dxi * dxi);
                O[4] = O[4] + pm * dyi * (dyi * dyi);
                O[5] = O[5] + pm * dyi * (dzi * dzi);
                O[6] = O[6] + pm * dzi * (dxi * dxi);
                O[7] = O[7] + pm * dzi * (dyi * dyi);
                O[8] = O[8] + pm * dzi * (dzi * dzi);
                O[9] = O[9] + pm * dxi * dyi * dzi;
            }
            if (oct && t->type[d] == 2) {
                O[0] = O[0] + 3.0 * dxi * Qd[0];
                O[1] = O[1] + 2.0 * dyi * Qd[3] + dxi * Qd[1];
                O[2] = O[2] + 2.0 * dzi * Qd[4] + dxi * Qd[2];
                O[3] = O[3] + 2.0 * dxi * Qd[3] + dyi * Qd[0];
                O[4] = O[4] + 3.0 * dyi * Qd[1];
                O[5] = O[5] + 2.0 * dzi * Qd[5] + dyi * Qd[2];
                O[6] = O[6] + 2.0 * dxi * Qd[4] + dzi * Qd[0];
                O[7] = O[7] + 2.0 * dyi * Qd[5] + dzi * Qd[1];
                O[8] = O[8] + 3.0 * dzi * Qd[2];
                O[9] = O[9] + dxi * Qd[5] + dyi * Qd[4] + dzi * Qd[3];
            }
        }
        if (oct) {
            double s = 0.0;
            for (int k = 0; k < 10; ++k) s += O[k];
            O[10] = s;
            O[11] = O[0] + O[1] + O[2];
            O[12] = O[3] + O[4] + O[5];
            O[13] = O[6] + O[7] + O[8];
        }
    }
}

/* octree_default.f90:1722-1809 (prepare_groups). */
static int prepare_groups(orc_octree *t) {
    int64_t nn = t->nnodes, n = t->n;
    t->count = (int32_t *)malloc((size_t)nn * 4 * sizeof(int32_t));
    t->order = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    t->gx = (double *)malloc((size_t)n * 4 * sizeof(double));
    if (!t->count || !t->order || !t->gx) return fail(ORC_ENOMEM, "groups: out of memory");
    t->first = t->count + nn; t->last = t->first + nn; t->groups = NULL;
    int32_t *groups = t->last + nn;
    t->gy = t->gx + n; t->gz = t->gy + n; t->gm = t->gz + n;
    for (int64_t node = nn - 1; node >= 0; --node) {
        if (t->type[node] == 1) {
            t->count[node] = t->particle[node] != -1;
        } else {
            int32_t k = 0;
            for (int i = 0; i < 8; ++i) {
                int64_t ch = t->child[8 * node + i];
                if (ch != -1) k += t->count[ch];
            }
            t->count[node] = k;
        }
    }
    if (t->count[0] != n) return fail(ORC_ELOST, "[prepare_groups] body lost");
    t->first[0] = 0;
    for (int64_t node = 0; node < nn; ++node) {
        int32_t k = t->first[node];
        if (t->type[node] == 1) {
            if (t->count[node] == 1) t->order[k] = t->particle[node];
        } else {
            for (int i = 0; i < 8; ++i) {
                int64_t ch = t->child[8 * node + i];
                if (ch == -1) continue;
                t->first[ch] = k;
                k += t->count[ch];
            }
        }
        t->last[node] = t->first[node] + t->count[node] - 1;
    }
    for (int64_t i = 0; i < n; ++i) {
        int32_t p = t->order[i];
        t->gm[i] = t->m[p]; t->gx[i] = t->x[p]; t->gy[i] = t->y[p]; t->gz[i] = t->z[p];
    }
    int32_t *stack = (int32_t *)malloc((size_t)(8 * (t->max_depth + 2) + 8) * sizeof(int32_t));
    if (!stack) return fail(ORC_ENOMEM, "groups: out of memory");
    int64_t ng = 0;
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
        int32_t node = stack[--top];
        if (t->count[node] == 0) continue;
        if (t->count[node] <= t->group_size || t->type[node] == 1) {
            groups[ng++] = node;
        } else {
            for (int i = 0; i < 8; ++i) {
                int32_t ch = t->child[8 * node + i];
                if (ch == -1) continue;
                stack[top++] = ch;
            }
        }
    }
    free(stack);
    t->ngroups = ng;
    t->groups = groups;
    return ORC_OK;
}

/* octree_default.f90:320-387 (init). */
int orc_octree_init(orc_octree *t, const double *x, const double *y, const double *z) {
    int64_t n = t->n;
    memcpy(t->x, x, (size_t)n * sizeof(double));
    memcpy(t->y, y, (size_t)n * sizeof(double));
    memcpy(t->z, z, (size_t)n * sizeof(double));
    t->nnodes = 0; t->most_depth = 0; t->err = 0;
    memset(t->quad, 0, (size_t)t->cap * 6 * sizeof(double));
    memset(t->oct, 0, (size_t)t->cap * 14 * sizeof(double));
    double info[4];
    system_size_info(n, x, y, z, info);
    int64_t root = add_node(t, info[0], info[1], info[2], t->side_amp * info[3], 0);
    (void)root;
    for (int64_t p = 0; p < n; ++p) add(t, 0, p);
    if (t->err) return fail(ORC_ECAPACITY, "INSUFFICIENT NUMBER OF NODES");
    if (t->multipole == 1) incorporate_particles(t);
    else evaluate_multipole(t);
    if (t->method >= 30) return prepare_groups(t);
    return ORC_OK;
}

int orc_octree_info(const orc_octree *t, int64_t *nnodes, int *most_depth, int64_t *ngroups) {
    if (nnodes) *nnodes = t->nnodes;
    if (most_depth) *most_depth = t->most_depth;
    if (ngroups) *ngroups = t->ngroups;
    return ORC_OK;
}

int orc_octree_get_nodes(const orc_octree *t, double *center3, double *halfside, double *L2,
                         double *mass, double *qcm3, int32_t *particle, int32_t *type,
                         int32_t *child8, int32_t *depth, double *quad6, double *oct14) {
    int64_t nn = t->nnodes;
    for (int64_t i = 0; i < nn; ++i) {
        if (center3) { center3[3 * i] = t->cx[i]; center3[3 * i + 1] = t->cy[i]; center3[3 * i + 2] = t->cz[i]; }
        if (qcm3) { qcm3[3 * i] = t->qx[i]; qcm3[3 * i + 1] = t->qy[i]; qcm3[3 * i + 2] = t->qz[i]; }
    }
    if (halfside) memcpy(halfside, t->halfside, (size_t)nn * sizeof(double));
    if (L2) memcpy(L2, t->L2, (size_t)nn * sizeof(double));
    if (mass) memcpy(mass, t->mass, (size_t)nn * sizeof(double));
    if (particle) memcpy(particle, t->particle, (size_t)nn * sizeof(int32_t));
    if (type) memcpy(type, t->type, (size_t)nn * sizeof(int32_t));
    if (child8) memcpy(child8, t->child, (size_t)nn * 8 * sizeof(int32_t));
    if (depth) memcpy(depth, t->depth, (size_t)nn * sizeof(int32_t));
    if (quad6) memcpy(quad6, t->quad, (size_t)nn * 6 * sizeof(double));
    if (oct14) memcpy(oct14, t->oct, (size_t)nn * 14 * sizeof(double));
    return ORC_OK;
}

/* octree_default.f90:895-1078 (bh_forces_over_p): DFS with an explicit stack. */
static void octree_walk(const orc_octree *t, int64_t p, double theta2, double G, double eps2,
                        int32_t *stack, double f[3], int64_t cnt[2]) {
    double pm = t->m[p], px = t->x[p], py = t->y[p], pz = t->z[p];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    int64_t npp = 0, npc = 0;
    int64_t top = 0;
    stack[top++] = 0;
    while (top > 0) {
        int64_t node = stack[--top];
        if (t->mass[node] == 0.0) continue;
        if (t->type[node] == 1 && t->particle[node] == p) continue;
        double dx = t->qx[node] - px, dy = t->qy[node] - py, dz = t->qz[node] - pz;
        double dist2 = dx * dx + dy * dy + dz * dz;
        double L2 = t->L2[node];
        if (t->type[node] == 1 || L2 <= theta2 * dist2 || t->depth[node] == t->max_depth) {
            if (t->type[node] == 1 || t->multipole == 1) {
                double rinv = 1.0 / sqrt(dist2 + eps2);
                rinv = rinv * rinv * rinv;
                double ff = G * pm * t->mass[node] * rinv;
                fx = fx + ff * dx; fy = fy + ff * dy; fz = fz + ff * dz;
                if (t->type[node] == 1) npp++; else npc++;
            } else {
                const double *q = t->quad + 6 * node, *o = t->oct + 14 * node;
                double invR = 1.0 / sqrt(dist2 + eps2);
                double invR2 = 1.0 / (dist2 + eps2);
                double invR3 = invR * invR2;
                double invR5 = invR3 * invR * invR;
                double invR7 = invR5 * invR * invR;
                double invR9 = invR7 * invR * invR;
                double Mx = dx * invR3 * t->mass[node];
                double My = dy * invR3 * t->mass[node];
                double Mz = dz * invR3 * t->mass[node];
                double mxi2 = q[0], myi2 = q[1], mzi2 = q[2], mxyi = q[3], mxzi = q[4], myzi = q[5];
                double dx2 = 15.0 * dx * dx * invR2 - 3.0;
                double dy2 = 15.0 * dy * dy * invR2 - 3.0;
                double dz2 = 15.0 * dz * dz * invR2 - 3.0;
                double dxyz = 15.0 * dx * dy * dz * invR2;
                double Qx = (mxi2 * (dx2 - 6.0) + myi2 * dy2 + mzi2 * dz2) * 0.5 * dx;
                double Qy = (myi2 * (dy2 - 6.0) + mzi2 * dz2 + mxi2 * dx2) * 0.5 * dy;
                double Qz = (mzi2 * (dz2 - 6.0) + mxi2 * dx2 + myi2 * dy2) * 0.5 * dz;
                Qx = Qx + mxyi * dy * dx2 + mxzi * dz * dx2 + myzi * dxyz;
                Qy = Qy + myzi * dz * dy2 + mxyi * dx * dy2 + mxzi * dxyz;
                Qz = Qz + mxzi * dx * dz2 + myzi * dy * dz2 + mxyi * dxyz;
                if (t->multipole == 4) {
                    fx = fx + G * pm * (Mx + invR5 * Qx);
                    fy = fy + G * pm * (My + invR5 * Qy);
                    fz = fz + G * pm * (Mz + invR5 * Qz);
                } else {                                         /* :1012-1063 */
                    double Ox = -1.5 * invR5 * o[11];
                    double Oy = -1.5 * invR5 * o[12];
                    double Oz = -1.5 * invR5 * o[13];
                    double Oc = 7.5 * invR7 * (dx * o[11] + dy * o[12] + dz * o[13]);
                    Ox = Ox + dx * Oc; Oy = Oy + dy * Oc; Oz = Oz + dz * Oc;
                    double ddx = dx * dx, ddy = dy * dy, ddz = dz * dz;
                    Ox = Ox + 7.5 * invR7 * (ddx * o[0] + ddy * o[1] + ddz * o[2] + 2.0 * dx * dy * o[3] +
                                             2.0 * dx * dz * o[6] + 2.0 * dy * dz * o[9]);
                    Oy = Oy + 7.5 * invR7 * (ddx * o[3] + ddy * o[4] + ddz * o[5] + 2.0 * dx * dy * o[1] +
                                             2.0 * dx * dz * o[9] + 2.0 * dy * dz * o[7]);
                    Oz = Oz + 7.5 * invR7 * (ddx * o[6] + ddy * o[7] + ddz * o[8] + 2.0 * dx * dy * o[9] +
                                             2.0 * dx * dz * o[2] + 2.0 * dy * dz * o[5]);
                    Oc = -17.5 * invR9 *
                         (ddx * dx * o[0] + ddy * dy * o[4] + ddz * dz * o[8] + 3.0 * ddx * dy * o[3] +
                          3.0 * ddx * dz * o[6] + 3.0 * ddy * dx * o[1] + 3.0 * ddy * dz * o[7] +
                          3.0 * ddz * dx * o[2] + 3.0 * ddz * dy * o[5] + 6.0 * dx * dy * dz * o[9]);
                    Ox = Ox + dx * Oc; Oy = Oy + dy * Oc; Oz = Oz + dz * Oc;
                    fx = fx + G * pm * (Mx + invR5 * Qx + Ox);
                    fy = fy + G * pm * (My + invR5 * Qy + Oy);
                    fz = fz + G * pm * (Mz + invR5 * Qz + Oz);
                }
                npc++;
            }
        } else {
            for (int i = 0; i < 8; ++i) {
                int32_t ch = t->child[8 * node + i];
                if (ch != -1) stack[top++] = ch;
            }
        }
    }
    f[0] = fx; f[1] = fy; f[2] = fz;
    if (cnt) { cnt[0] = npp; cnt[1] = npc; }
}

static double maxd(double a, double b) { return a > b ? a : b; }

/* octree_default.f90:1833-2095 (group_worker) for one group. */
static void group_forces(const orc_octree *t, int64_t gi, double theta2, double G, double eps2,
                         double *out, int64_t **sbuf, int64_t *scap, double **cbuf, int64_t *ccap,
                         int32_t *stack) {
    int64_t n = t->n;
    int mpole = t->multipole;
    int ncd = mpole == 1 ? 4 : (mpole == 4 ? 10 : 24);
    int32_t g = t->groups[gi];
    int32_t gf = t->first[g], gl = t->last[g];
    double h = t->halfside[g];
    double gmin[3] = {t->cx[g] - h, t->cy[g] - h, t->cz[g] - h};
    double gmax[3] = {t->cx[g] + h, t->cy[g] + h, t->cz[g] + h};
    int64_t ns = 0, nc = 0;
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
        int32_t node = stack[--top];
        if (node == g) continue;
        if (t->mass[node] == 0.0) continue;
        if (t->first[node] <= gf && t->last[node] >= gl) {
            for (int i = 0; i < 8; ++i) {
                int32_t ch = t->child[8 * node + i];
                if (ch != -1) stack[top++] = ch;
            }
            continue;
        }
        if (t->type[node] == 1) {
            for (int32_t a = t->first[node]; a <= t->last[node]; ++a) {
                if (ns >= *scap) { *scap *= 2; *sbuf = (int64_t *)realloc(*sbuf, (size_t)*scap * sizeof(int64_t)); }
                (*sbuf)[ns++] = a;
            }
            continue;
        }
        double cc[3] = {t->qx[node], t->qy[node], t->qz[node]};
        double dist2 = 0.0;
        for (int i = 0; i < 3; ++i) {
            double dd = maxd(maxd(gmin[i] - cc[i], 0.0), cc[i] - gmax[i]);
            dist2 = dist2 + dd * dd;
        }
        if (t->L2[node] <= theta2 * dist2 || t->depth[node] >= t->max_depth) {
            if (nc >= *ccap) { *ccap *= 2; *cbuf = (double *)realloc(*cbuf, (size_t)*ccap * 24 * sizeof(double)); }
            double *cd = *cbuf + 24 * nc;
            cd[0] = t->mass[node]; cd[1] = cc[0]; cd[2] = cc[1]; cd[3] = cc[2];
            if (mpole >= 4) for (int k = 0; k < 6; ++k) cd[4 + k] = t->quad[6 * node + k];
            if (mpole >= 8) for (int k = 0; k < 14; ++k) cd[10 + k] = t->oct[14 * node + k];
            nc++;
        } else {
            for (int i = 0; i < 8; ++i) {
                int32_t ch = t->child[8 * node + i];
                if (ch != -1) stack[top++] = ch;
            }
        }
    }
    (void)ncd;
    const int64_t *sl = *sbuf;
    for (int32_t i = gf; i <= gl; ++i) {
        double xi = t->gx[i], yi = t->gy[i], zi = t->gz[i];
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int32_t j = gf; j <= gl; ++j) {
            if (j == i) continue;
            double dx = t->gx[j] - xi, dy = t->gy[j] - yi, dz = t->gz[j] - zi;
            double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            double invr = 1.0 / sqrt(dist2);
            double invr3 = invr * invr * invr;
            double ff = t->gm[j] * invr3;
            ax = ax + ff * dx; ay = ay + ff * dy; az = az + ff * dz;
        }
        for (int64_t s = 0; s < ns; ++s) {
            int64_t j = sl[s];
            double dx = t->gx[j] - xi, dy = t->gy[j] - yi, dz = t->gz[j] - zi;
            double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            double invr = 1.0 / sqrt(dist2);
            double invr3 = invr * invr * invr;
            double ff = t->gm[j] * invr3;
            ax = ax + ff * dx; ay = ay + ff * dy; az = az + ff * dz;
        }
        for (int64_t j = 0; j < nc; ++j) {
            const double *cd = *cbuf + 24 * j;
            double dx = cd[1] - xi, dy = cd[2] - yi, dz = cd[3] - zi;
            double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            double invr = 1.0 / sqrt(dist2);
            double invr3 = invr * invr * invr;
            if (mpole == 1) {
                double ff = cd[0] * invr3;
                ax = ax + ff * dx; ay = ay + ff * dy; az = az + ff * dz;
                continue;
            }
            double invr5 = invr3 * invr * invr;
            double invr7 = invr5 * invr * invr;
            double qx = cd[4] * dx + cd[7] * dy + cd[8] * dz;
            double qy = cd[7] * dx + cd[5] * dy + cd[9] * dz;
            double qz = cd[8] * dx + cd[9] * dy + cd[6] * dz;
            double dqd = dx * qx + dy * qy + dz * qz;
            double trq = cd[4] + cd[5] + cd[6];
            double s = cd[0] * invr3 - 1.5 * trq * invr5 + 7.5 * dqd * invr7;
            ax = ax + s * dx - 3.0 * qx * invr5;
            ay = ay + s * dy - 3.0 * qy * invr5;
            az = az + s * dz - 3.0 * qz * invr5;
            if (mpole == 8) {                                    /* :2055-2082 */
                double invr9 = invr7 * invr * invr;
                double oc = 7.5 * invr7 * (dx * cd[21] + dy * cd[22] + dz * cd[23]);
                double ox = -1.5 * invr5 * cd[21] + dx * oc;
                double oy = -1.5 * invr5 * cd[22] + dy * oc;
                double oz = -1.5 * invr5 * cd[23] + dz * oc;
                ox = ox + 7.5 * invr7 * (dx * dx * cd[10] + dy * dy * cd[11] + dz * dz * cd[12]);
                ox = ox + 15.0 * invr7 * (dx * dy * cd[13] + dx * dz * cd[16] + dy * dz * cd[19]);
                oy = oy + 7.5 * invr7 * (dx * dx * cd[13] + dy * dy * cd[14] + dz * dz * cd[15]);
                oy = oy + 15.0 * invr7 * (dx * dy * cd[11] + dx * dz * cd[19] + dy * dz * cd[17]);
                oz = oz + 7.5 * invr7 * (dx * dx * cd[16] + dy * dy * cd[17] + dz * dz * cd[18]);
                oz = oz + 15.0 * invr7 * (dx * dy * cd[19] + dx * dz * cd[12] + dy * dz * cd[15]);
                oc = dx * dx * dx * cd[10] + dy * dy * dy * cd[14] + dz * dz * dz * cd[18];
                oc = oc + 3.0 * (dx * dx * dy * cd[13] + dx * dx * dz * cd[16] + dx * dy * dy * cd[11]);
                oc = oc + 3.0 * (dy * dy * dz * cd[17] + dx * dz * dz * cd[12] + dy * dz * dz * cd[15]);
                oc = oc + 6.0 * dx * dy * dz * cd[19];
                oc = -17.5 * invr9 * oc;
                ox = ox + dx * oc; oy = oy + dy * oc; oz = oz + dz * oc;
                ax = ax + ox; ay = ay + oy; az = az + oz;
            }
        }
        int32_t k = t->order[i];
        out[k] = G * t->gm[i] * ax;
        out[n + k] = G * t->gm[i] * ay;
        out[2 * n + k] = G * t->gm[i] * az;
    }
}

/* Forces for all particles, ORIGINAL order, SoA out.  Methods 10-12 follow
 * test_forces.f90:201-211 (per-particle loop), 30-32 follow forces_groups
 * (octree_default.f90:1811-1831). */
static int octree_dehnen(const orc_octree *t, double theta2, double G, double eps2, double *out);

int orc_octree_forces(const orc_octree *t, double theta2, double G, double eps2, double *out,
                      int nthreads) {
    int64_t n = t->n;
    if (t->method >= 20 && t->method < 30) return octree_dehnen(t, theta2, G, eps2, out);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    if (t->method < 30) {
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
        {
            int32_t *stack = (int32_t *)malloc((size_t)(t->nnodes + 8) * sizeof(int32_t));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
            for (int64_t p = 0; p < n; ++p) {
                double f[3];
                octree_walk(t, p, theta2, G, eps2, stack, f, NULL);
                out[p] = f[0]; out[n + p] = f[1]; out[2 * n + p] = f[2];
            }
            free(stack);
        }
    } else {
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
        {
            int64_t scap = 2048, ccap = 512;
            int64_t *sbuf = (int64_t *)malloc((size_t)scap * sizeof(int64_t));
            double *cbuf = (double *)malloc((size_t)ccap * 24 * sizeof(double));
            int32_t *stack = (int32_t *)malloc((size_t)(8 * (t->max_depth + 2) + 8) * sizeof(int32_t));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int64_t g = 0; g < t->ngroups; ++g)
                group_forces(t, g, theta2, G, eps2, out, &sbuf, &scap, &cbuf, &ccap, stack);
            free(sbuf); free(cbuf); free(stack);
        }
    }
    (void)nthreads;
    return ORC_OK;
}

/* Per-particle walk (methods 10-12) on a subset of targets; counts optional. */
int orc_octree_forces_targets(const orc_octree *t, double theta2, double G, double eps2,
                              int64_t nt, const int64_t *targets, double *out, int64_t *counts,
                              int nthreads) {
    if (t->method >= 20) return fail(ORC_EINVAL, "targets: per-particle methods only");
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        int32_t *stack = (int32_t *)malloc((size_t)(t->nnodes + 8) * sizeof(int32_t));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
        for (int64_t k = 0; k < nt; ++k) {
            double f[3];
            int64_t c[2];
            octree_walk(t, targets[k], theta2, G, eps2, stack, f, c);
            out[k] = f[0]; out[nt + k] = f[1]; out[2 * nt + k] = f[2];
            if (counts) { counts[2 * k] = c[0]; counts[2 * k + 1] = c[1]; }
        }
        free(stack);
    }
    (void)nthreads;
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* FP64 direct sum (fortran/direct_forces.f90)                                */
/* ------------------------------------------------------------------------- */

/* direct_forces.f90:18-38: sequential pair loop with Newton's third law. */
int orc_direct_forces(int64_t n, const double *m, const double *x, const double *y,
                      const double *z, double G, double eps2, double *out) {
    memset(out, 0, (size_t)n * 3 * sizeof(double));
    double *fx = out, *fy = out + n, *fz = out + 2 * n;
    for (int64_t a = 1; a < n; ++a) {
        for (int64_t b = 0; b < a; ++b) {
            double dx = x[b] - x[a], dy = y[b] - y[a], dz = z[b] - z[a];
            double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            double dist = sqrt(dist2);
            double f = G * m[a] * m[b] / (dist * dist2);
            fx[a] = fx[a] + f * dx; fy[a] = fy[a] + f * dy; fz[a] = fz[a] + f * dz;
            fx[b] = fx[b] - f * dx; fy[b] = fy[b] - f * dy; fz[b] = fz[b] - f * dz;
        }
    }
    return ORC_OK;
}

/* The same pair force summed for a subset of targets (original indices), in
 * source order 0..n-1 skipping the target itself. */
int orc_direct_forces_targets(int64_t n, const double *m, const double *x, const double *y,
                              const double *z, double G, double eps2, int64_t nt,
                              const int64_t *targets, double *out, int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
    for (int64_t k = 0; k < nt; ++k) {
        int64_t a = targets[k];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int64_t b = 0; b < n; ++b) {
            if (b == a) continue;
            double dx = x[b] - x[a], dy = y[b] - y[a], dz = z[b] - z[a];
            double dist2 = dx * dx + dy * dy + dz * dz + eps2;
            double dist = sqrt(dist2);
            double f = G * m[a] * m[b] / (dist * dist2);
            fx = fx + f * dx; fy = fy + f * dy; fz = fz + f * dz;
        }
        out[k] = fx; out[nt + k] = fy; out[2 * nt + k] = fz;
    }
    (void)nthreads;
    return ORC_OK;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* Dehnen's dual-tree method, fortran/octree_default.f90:1095-1712 (methods
 * 20/21/22): evaluate_rmax (:1095-1131), mutual_interaction_walk_sequential
 * (:1133-1247), the mutual interactions (monopole :1425-1445; quadrupole
 * :1447-1558, with the octupole torque term for multipole 8) and dehnen_forces
 * (:1560-1673, the downward pass).  It runs over a generic view of a tree --
 * entities in parent-before-child order with CSR child lists -- so the same
 * code serves the insertion tree (the reference's own) and the Morton tree
 * (whose topology the device build reproduces).  Forces are G m a, SoA
 * (x block, y block, z block) in the particles' output order. */

typedef struct {
    int64_t ne;
    int64_t *cbeg;      /* ne + 1 */
    int32_t *clist;
    int32_t *leaf;      /* 1: a particle leaf (ns_type == 1) */
    int64_t *particle;  /* output index of a leaf's particle, -1 none */
    double *mass, *cx, *cy, *cz;
    double *quad;       /* 6 per entity (multipole >= 4), raw moments about the COM */
    double *oct;        /* 14 per entity (multipole >= 8), octree_default layout */
} dtree;

static void dtree_free(dtree *t) {
    free(t->cbeg); free(t->clist); free(t->leaf); free(t->particle);
    free(t->mass); free(t->quad); free(t->oct);
}

static int dtree_alloc(dtree *t, int64_t ne, int64_t nlinks) {
    memset(t, 0, sizeof *t);
    t->ne = ne;
    t->cbeg = (int64_t *)calloc((size_t)ne + 1, sizeof(int64_t));
    t->clist = (int32_t *)malloc((size_t)(nlinks > 0 ? nlinks : 1) * sizeof(int32_t));
    t->leaf = (int32_t *)calloc((size_t)ne, sizeof(int32_t));
    t->particle = (int64_t *)malloc((size_t)ne * sizeof(int64_t));
    t->mass = (double *)calloc((size_t)ne * 4, sizeof(double));
    t->quad = (double *)calloc((size_t)ne * 6, sizeof(double));
    t->oct = (double *)calloc((size_t)ne * 14, sizeof(double));
    if (!t->cbeg || !t->clist || !t->leaf || !t->particle || !t->mass || !t->quad || !t->oct) {
        dtree_free(t);
        return fail(ORC_ENOMEM, "dehnen: out of memory");
    }
    t->cx = t->mass + ne; t->cy = t->cx + ne; t->cz = t->cy + ne;
    return ORC_OK;
}

/* ind_oct of octree_default.f90:233-241, 0-based: component of O_jkl */
static const int IND_OCT[3][3][3] = {
    {{0, 3, 6}, {3, 1, 9}, {6, 9, 2}},
    {{3, 1, 9}, {1, 4, 7}, {9, 7, 5}},
    {{6, 9, 2}, {9, 7, 5}, {2, 5, 8}}};

/* :1095-1131 */
static void dehnen_rmax(const dtree *t, double *rmax) {
    for (int64_t e = t->ne - 1; e >= 0; --e) {
        rmax[e] = 0.0;
        if (t->leaf[e]) continue;
        double r = 0.0;
        for (int64_t k = t->cbeg[e]; k < t->cbeg[e + 1]; ++k) {
            int64_t c = t->clist[k];
            if (t->mass[c] == 0.0) continue;
            double dx = t->cx[c] - t->cx[e];
            double dy = t->cy[c] - t->cy[e];
            double dz = t->cz[c] - t->cz[e];
            double dist = sqrt(dx * dx + dy * dy + dz * dz);
            double v = dist + rmax[c];
            if (v > r) r = v;
        }
        rmax[e] = r;
    }
}

/* :1425-1445 (monopole) and :1447-1558 (quadrupole, octupole torque term),
 * accumulated into both nodes as :1200-1221 does. */
static void dehnen_mutual(const dtree *t, int mult, int64_t a, int64_t b, double G, double eps2,
                          double *F, double *H, double *T) {
    const double Ma = t->mass[a], Mb = t->mass[b];
    if (mult == 1) {
        double dx = t->cx[b] - t->cx[a];
        double dy = t->cy[b] - t->cy[a];
        double dz = t->cz[b] - t->cz[a];
        double dist2 = dx * dx + dy * dy + dz * dz;
        double rinv3 = 1.0 / pow(dist2 + eps2, 1.5);
        double factor = G * rinv3;
        double f[3] = {factor * dx, factor * dy, factor * dz};
        for (int k = 0; k < 3; ++k) {
            F[3 * a + k] = F[3 * a + k] + Mb * f[k];
            F[3 * b + k] = F[3 * b + k] - Ma * f[k];
        }
        return;
    }
    double dx = t->cx[a] - t->cx[b];
    double dy = t->cy[a] - t->cy[b];
    double dz = t->cz[a] - t->cz[b];
    double r2 = dx * dx + dy * dy + dz * dz + eps2;
    double rinv3 = 1.0 / pow(r2, 1.5);
    double rinv5 = 1.0 / pow(r2, 2.5);
    double rinv7 = 1.0 / pow(r2, 3.5);
    double D1[3], D2[6], D3[10];
    D1[0] = -G * dx * rinv3;
    D1[1] = -G * dy * rinv3;
    D1[2] = -G * dz * rinv3;
    D2[0] = G * (3.0 * dx * dx * rinv5 - rinv3);
    D2[1] = G * (3.0 * dy * dy * rinv5 - rinv3);
    D2[2] = G * (3.0 * dz * dz * rinv5 - rinv3);
    D2[3] = G * 3.0 * dx * dy * rinv5;
    D2[4] = G * 3.0 * dx * dz * rinv5;
    D2[5] = G * 3.0 * dy * dz * rinv5;
    D3[0] = G * (-15.0 * dx * dx * dx * rinv7 + 9.0 * dx * rinv5);
    D3[1] = G * (-15.0 * dx * dx * dy * rinv7 + 3.0 * dy * rinv5);
    D3[2] = G * (-15.0 * dx * dx * dz * rinv7 + 3.0 * dz * rinv5);
    D3[3] = G * (-15.0 * dx * dy * dy * rinv7 + 3.0 * dx * rinv5);
    D3[4] = G * (-15.0 * dx * dy * dz * rinv7);
    D3[5] = G * (-15.0 * dx * dz * dz * rinv7 + 3.0 * dx * rinv5);
    D3[6] = G * (-15.0 * dy * dy * dy * rinv7 + 9.0 * dy * rinv5);
    D3[7] = G * (-15.0 * dy * dy * dz * rinv7 + 3.0 * dz * rinv5);
    D3[8] = G * (-15.0 * dy * dz * dz * rinv7 + 3.0 * dy * rinv5);
    D3[9] = G * (-15.0 * dz * dz * dz * rinv7 + 9.0 * dz * rinv5);
    double Qa[6], Qb[6];
    for (int k = 0; k < 6; ++k) { Qa[k] = t->quad[6 * a + k] / Ma; Qb[k] = t->quad[6 * b + k] / Mb; }
    double CQa[3], CQb[3];
    CQa[0] = Qa[0] * D3[0] + 2.0 * Qa[3] * D3[1] + 2.0 * Qa[4] * D3[2] + Qa[1] * D3[3] +
             2.0 * Qa[5] * D3[4] + Qa[2] * D3[5];
    CQb[0] = Qb[0] * D3[0] + 2.0 * Qb[3] * D3[1] + 2.0 * Qb[4] * D3[2] + Qb[1] * D3[3] +
             2.0 * Qb[5] * D3[4] + Qb[2] * D3[5];
    CQa[1] = Qa[0] * D3[1] + 2.0 * Qa[3] * D3[3] + 2.0 * Qa[4] * D3[4] + Qa[1] * D3[6] +
             2.0 * Qa[5] * D3[7] + Qa[2] * D3[8];
    CQb[1] = Qb[0] * D3[1] + 2.0 * Qb[3] * D3[3] + 2.0 * Qb[4] * D3[4] + Qb[1] * D3[6] +
             2.0 * Qb[5] * D3[7] + Qb[2] * D3[8];
    CQa[2] = Qa[0] * D3[2] + 2.0 * Qa[3] * D3[4] + 2.0 * Qa[4] * D3[5] + Qa[1] * D3[7] +
             2.0 * Qa[5] * D3[8] + Qa[2] * D3[9];
    CQb[2] = Qb[0] * D3[2] + 2.0 * Qb[3] * D3[4] + 2.0 * Qb[4] * D3[5] + Qb[1] * D3[7] +
             2.0 * Qb[5] * D3[8] + Qb[2] * D3[9];
    double fa[3], fb[3], fc[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 3; ++k) {
        fa[k] = Mb * (D1[k] + 0.5 * CQb[k]);
        fb[k] = -Ma * (D1[k] + 0.5 * CQa[k]);
    }
    if (mult >= 8) {
        double R[3] = {dx, dy, dz}, ci[3] = {0, 0, 0}, CRR[3] = {0, 0, 0};
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) {
                    double Cjkl = Mb * t->oct[14 * a + IND_OCT[j][k][l]] -
                                  Ma * t->oct[14 * b + IND_OCT[j][k][l]];
                    if (k == l) ci[j] = ci[j] + Cjkl;
                    CRR[j] = CRR[j] + Cjkl * R[k] * R[l];
                }
        for (int k = 0; k < 3; ++k)
            fc[k] = 0.5 * (3.0 * G * rinv5 * ci[k] - 15.0 * G * rinv7 * CRR[k]);
    }
    for (int k = 0; k < 3; ++k) {
        F[3 * a + k] = F[3 * a + k] + fa[k] + fc[k] / Ma;
        F[3 * b + k] = F[3 * b + k] + fb[k] - fc[k] / Mb;
    }
    for (int k = 0; k < 6; ++k) {
        H[6 * a + k] = H[6 * a + k] + Mb * D2[k];
        H[6 * b + k] = H[6 * b + k] + Ma * D2[k];
    }
    for (int k = 0; k < 10; ++k) {
        T[10 * a + k] = T[10 * a + k] + Mb * D3[k];
        T[10 * b + k] = T[10 * b + k] - Ma * D3[k];
    }
}

/* The whole method on entity 0 as the root.  *pairs (optional) returns the
 * number of mutual interactions. */
static int dehnen_run(const dtree *t, int mult, double theta2, double G, double eps2, int64_t n,
                      double *out, int64_t *pairs) {
    const int64_t ne = t->ne;
    double *rmax = (double *)malloc((size_t)ne * sizeof(double));
    double *F = (double *)calloc((size_t)ne * 3, sizeof(double));
    double *H = (double *)calloc((size_t)ne * 6, sizeof(double));
    double *T = (double *)calloc((size_t)ne * 10, sizeof(double));
    int64_t cap = 36 * ne + 64, top = 0, np = 0;
    int64_t *st = (int64_t *)malloc((size_t)cap * 2 * sizeof(int64_t));
    if (!rmax || !F || !H || !T || !st) {
        free(rmax); free(F); free(H); free(T); free(st);
        return fail(ORC_ENOMEM, "dehnen: out of memory");
    }
    for (int64_t i = 0; i < 3 * n; ++i) out[i] = 0.0;
    dehnen_rmax(t, rmax);
#define PUSH(A, B)                                                                  \
    do {                                                                            \
        if (top == cap) {                                                           \
            cap *= 2;                                                               \
            int64_t *ns = (int64_t *)realloc(st, (size_t)cap * 2 * sizeof(int64_t)); \
            if (!ns) { free(st); st = NULL; goto oom; }                              \
            st = ns;                                                                \
        }                                                                           \
        st[2 * top] = (A); st[2 * top + 1] = (B); ++top;                            \
    } while (0)
    PUSH(0, 0);
    while (top > 0) {
        --top;
        const int64_t a = st[2 * top], b = st[2 * top + 1];
        if (t->mass[a] == 0.0) continue;
        if (t->mass[b] == 0.0) continue;
        if (a == b) {
            if (t->leaf[a]) continue;
            for (int64_t i = t->cbeg[a]; i < t->cbeg[a + 1]; ++i)
                for (int64_t j = i; j < t->cbeg[a + 1]; ++j) PUSH(t->clist[i], t->clist[j]);
            continue;
        }
        double dx = t->cx[a] - t->cx[b];
        double dy = t->cy[a] - t->cy[b];
        double dz = t->cz[a] - t->cz[b];
        double dist2 = dx * dx + dy * dy + dz * dz;
        double rs = rmax[a] + rmax[b];
        double rsum2 = rs * rs;
        if (rsum2 <= theta2 * dist2) {
            dehnen_mutual(t, mult, a, b, G, eps2, F, H, T);
            ++np;
            continue;
        }
        if (rmax[a] >= rmax[b]) {
            for (int64_t i = t->cbeg[a]; i < t->cbeg[a + 1]; ++i) PUSH(t->clist[i], b);
        } else {
            for (int64_t i = t->cbeg[b]; i < t->cbeg[b + 1]; ++i) PUSH(a, t->clist[i]);
        }
    }
#undef PUSH
    /* :1560-1673 downward pass */
    for (int64_t e = 0; e < ne; ++e) {
        if (t->leaf[e]) continue;
        const double *h = H + 6 * e, *tt = T + 10 * e;
        for (int64_t k = t->cbeg[e]; k < t->cbeg[e + 1]; ++k) {
            const int64_t c = t->clist[k];
            if (t->mass[c] == 0.0) continue;
            double fch[3];
            for (int q = 0; q < 3; ++q) fch[q] = F[3 * c + q] + F[3 * e + q];
            if (mult >= 4) {
                double dx = t->cx[c] - t->cx[e];
                double dy = t->cy[c] - t->cy[e];
                double dz = t->cz[c] - t->cz[e];
                const double hxx = h[0], hyy = h[1], hzz = h[2], hxy = h[3], hxz = h[4], hyz = h[5];
                const double txxx = tt[0], txxy = tt[1], txxz = tt[2], txyy = tt[3], txyz = tt[4],
                             txzz = tt[5], tyyy = tt[6], tyyz = tt[7], tyzz = tt[8], tzzz = tt[9];
                fch[0] = fch[0] + hxx * dx + hxy * dy + hxz * dz + txxy * dx * dy + txxz * dx * dz +
                         txyz * dy * dz + 0.5 * (txxx * dx * dx + txyy * dy * dy + txzz * dz * dz);
                fch[1] = fch[1] + hxy * dx + hyy * dy + hyz * dz + txyy * dx * dy + txyz * dx * dz +
                         tyyz * dy * dz + 0.5 * (txxy * dx * dx + tyyy * dy * dy + tyzz * dz * dz);
                fch[2] = fch[2] + hxz * dx + hyz * dy + hzz * dz + txyz * dx * dy + txzz * dx * dz +
                         tyzz * dy * dz + 0.5 * (txxz * dx * dx + tyyz * dy * dy + tzzz * dz * dz);
                if (!t->leaf[c]) {
                    double *hc = H + 6 * c;
                    hc[0] = hc[0] + hxx + txxx * dx + txxy * dy + txxz * dz;
                    hc[1] = hc[1] + hyy + txyy * dx + tyyy * dy + tyyz * dz;
                    hc[2] = hc[2] + hzz + txzz * dx + tyzz * dy + tzzz * dz;
                    hc[3] = hc[3] + hxy + txxy * dx + txyy * dy + txyz * dz;
                    hc[4] = hc[4] + hxz + txxz * dx + txyz * dy + txzz * dz;
                    hc[5] = hc[5] + hyz + txyz * dx + tyyz * dy + tyzz * dz;
                }
                for (int q = 0; q < 10; ++q) T[10 * c + q] = T[10 * c + q] + tt[q];
            }
            for (int q = 0; q < 3; ++q) F[3 * c + q] = fch[q];
            if (t->leaf[c]) {
                const int64_t p = t->particle[c];
                if (p < 0) continue;
                for (int q = 0; q < 3; ++q) out[q * n + p] = t->mass[c] * F[3 * c + q];
            }
        }
    }
    if (pairs) *pairs = np;
    free(rmax); free(F); free(H); free(T); free(st);
    return ORC_OK;
oom:
    free(rmax); free(F); free(H); free(T);
    return fail(ORC_ENOMEM, "dehnen: out of memory for the pair stack");
}

/* Insertion tree (octree_default) as a generic tree. */
static int octree_dehnen(const orc_octree *t, double theta2, double G, double eps2, double *out) {
    dtree d;
    int64_t links = 0;
    for (int64_t e = 0; e < t->nnodes; ++e)
        for (int c = 0; c < 8; ++c) links += t->child[8 * e + c] != -1;
    int rc = dtree_alloc(&d, t->nnodes, links);
    if (rc) return rc;
    int64_t k = 0;
    for (int64_t e = 0; e < t->nnodes; ++e) {
        d.cbeg[e] = k;
        for (int c = 0; c < 8; ++c)
            if (t->child[8 * e + c] != -1) d.clist[k++] = t->child[8 * e + c];
        d.leaf[e] = t->type[e] == 1;
        d.particle[e] = t->type[e] == 1 ? t->particle[e] : -1;
        d.mass[e] = t->mass[e]; d.cx[e] = t->qx[e]; d.cy[e] = t->qy[e]; d.cz[e] = t->qz[e];
        if (t->multipole >= 4) memcpy(d.quad + 6 * e, t->quad + 6 * e, 6 * sizeof(double));
        if (t->multipole >= 8) memcpy(d.oct + 14 * e, t->oct + 14 * e, 14 * sizeof(double));
    }
    d.cbeg[t->nnodes] = k;
    rc = dehnen_run(&d, t->multipole, theta2, G, eps2, t->n, out, NULL);
    dtree_free(&d);
    return rc;
}

/* Raw second and third moments of sorted particles [first, last] about c,
 * with the summary sums of octree_default.f90:875-880. */
static void direct_moments(const orc_morton *t, int64_t first, int64_t last, const double c[3],
                           double *Q, double *O) {
    for (int k = 0; k < 6; ++k) Q[k] = 0.0;
    for (int k = 0; k < 14; ++k) O[k] = 0.0;
    for (int64_t p = first; p <= last; ++p) {
        const double pm = t->ms[p];
        const double dx = t->qx[p] - c[0], dy = t->qy[p] - c[1], dz = t->qz[p] - c[2];
        Q[0] += pm * dx * dx; Q[1] += pm * dy * dy; Q[2] += pm * dz * dz;
        Q[3] += pm * dx * dy; Q[4] += pm * dx * dz; Q[5] += pm * dy * dz;
        O[0] += pm * dx * dx * dx; O[1] += pm * dx * dy * dy; O[2] += pm * dx * dz * dz;
        O[3] += pm * dy * dx * dx; O[4] += pm * dy * dy * dy; O[5] += pm * dy * dz * dz;
        O[6] += pm * dz * dx * dx; O[7] += pm * dz * dy * dy; O[8] += pm * dz * dz * dz;
        O[9] += pm * dx * dy * dz;
    }
    double s = 0.0;
    for (int k = 0; k < 10; ++k) s += O[k];
    O[10] = s;
    O[11] = O[0] + O[1] + O[2];
    O[12] = O[3] + O[4] + O[5];
    O[13] = O[6] + O[7] + O[8];
}

/* Morton tree (morton_octree.f90) as a generic tree: a node of one particle
 * is a particle leaf at its centre of mass; a depth-L node of several bodies
 * (identical keys) gets one particle leaf per body, appended after the nodes;
 * moments are summed directly over each node's bodies.  mult 1, 4 or 8. */
int orc_morton_dehnen(const orc_morton *t, double G, double eps2, double theta2, int mult,
                      double *out, int64_t *pairs) {
    if (mult != 1 && mult != 4 && mult != 8) return fail(ORC_EINVAL, "dehnen: mult must be 1, 4 or 8");
    const int64_t nn = t->nnodes;
    int64_t extra = 0, links = 0;
    for (int64_t e = 0; e < nn; ++e) {
        if (t->first[e] == t->last[e]) continue;
        if (t->nchild[e] == 0) { extra += t->last[e] - t->first[e] + 1; links += t->last[e] - t->first[e] + 1; }
        else links += t->nchild[e];
    }
    dtree d;
    int rc = dtree_alloc(&d, nn + extra, links);
    if (rc) return rc;
    int64_t k = 0, nx = nn;
    for (int64_t e = 0; e < nn; ++e) {
        d.cbeg[e] = k;
        d.mass[e] = t->nmass[e];
        d.cx[e] = t->qcm[3 * e]; d.cy[e] = t->qcm[3 * e + 1]; d.cz[e] = t->qcm[3 * e + 2];
        d.particle[e] = -1;
        if (t->first[e] == t->last[e]) {
            d.leaf[e] = 1;
            d.particle[e] = t->perm[t->first[e]];
            continue;
        }
        direct_moments(t, t->first[e], t->last[e], t->qcm + 3 * e, d.quad + 6 * e, d.oct + 14 * e);
        if (t->nchild[e] == 0) {
            for (int64_t p = t->first[e]; p <= t->last[e]; ++p) {
                d.clist[k++] = (int32_t)nx;
                d.leaf[nx] = 1;
                d.particle[nx] = t->perm[p];
                d.mass[nx] = t->ms[p];
                d.cx[nx] = t->qx[p]; d.cy[nx] = t->qy[p]; d.cz[nx] = t->qz[p];
                ++nx;
            }
        } else {
            for (int c = 0; c < t->nchild[e]; ++c) d.clist[k++] = t->child[8 * e + c];
        }
    }
    for (int64_t e = nn; e <= nn + extra; ++e) d.cbeg[e] = k;
    rc = dehnen_run(&d, mult, theta2, G, eps2, t->n, out, pairs);
    dtree_free(&d);
    return rc;
}
