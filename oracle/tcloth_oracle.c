/*
 * tcloth_oracle.c -- CPU oracle (test infrastructure only) for the XPBD
 * cloth substep of Taremin/TareminCloth's cloth_core.
 *
 * A sequential restatement of the reference algorithm.  Compiled with
 * -ffp-contract=off so each float operation rounds exactly as written; the
 * order of every float expression follows the reference WGSL so that the
 * CUDA product (built with --fmad=false and IEEE div/sqrt) can be compared
 * bit for bit.  Integer accumulations that the reference does with atomics
 * are plain (wrapping) integer sums here: they do not depend on order.
 *
 * Where the reference is nondeterministic (the atomic scatter of the
 * counting-sort hash, spatial_grid_sort.wgsl:182-194) the oracle uses the
 * canonical order: ascending vertex / edge index within a hash bucket.
 *
 * Out of scope here (not reached by the workloads): sewing priority,
 * coarse constraints, pair-cache and virtual-particle self-collision, edge
 * colliders.  Where the reference takes the two edges of a sewn seam in
 * hash-map order (mesh.rs:742-765), the oracle takes them in face order;
 * the resulting constraint acts the same either way round.
 */
#include "tcloth_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } v3;

static inline v3 V3(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline v3 vdiv(v3 a, float s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlen(v3 a) { return sqrtf(vdot(a, a)); }
static inline float fminx(float a, float b) { return fminf(a, b); }
static inline float fmaxx(float a, float b) { return fmaxf(a, b); }
static inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
static inline v3 vmin(v3 a, v3 b) { return V3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
static inline v3 vmax(v3 a, v3 b) { return V3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
/* WGSL mix(a, b, t) = a * (1 - t) + b * t */
static inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
static inline v3 vmix(v3 a, v3 b, float t) {
    float u = 1.0f - t;
    return V3(a.x * u + b.x * t, a.y * u + b.y * t, a.z * u + b.z * t);
}
/* f32 -> i32 conversion of an already floored value: saturating, NaN -> 0 */
static inline int32_t f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483647.0f) return INT32_MAX;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}
static inline float lenv(const float *a) { return sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

static const float EPS = 1e-7f;

/* ------------------------------------------------------------------ */
/* small containers                                                    */
/* ------------------------------------------------------------------ */
typedef struct { uint64_t *keys; uint32_t cap, n; } KSet;
static void kset_init(KSet *s, uint32_t expect) {
    uint32_t c = 16;
    while (c < expect * 2 + 16) c <<= 1;
    s->cap = c; s->n = 0;
    s->keys = (uint64_t *)malloc(sizeof(uint64_t) * c);
    memset(s->keys, 0xff, sizeof(uint64_t) * c);
}
static void kset_free(KSet *s) { free(s->keys); s->keys = NULL; }
static uint32_t kmix(uint64_t k) {
    k ^= k >> 33; k *= 0xff51afd7ed558ccdULL; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ULL; k ^= k >> 33;
    return (uint32_t)k;
}
static int kset_has(const KSet *s, uint64_t k) {
    uint32_t m = s->cap - 1, h = kmix(k) & m;
    while (s->keys[h] != UINT64_MAX) { if (s->keys[h] == k) return 1; h = (h + 1) & m; }
    return 0;
}
static void kset_grow(KSet *s);
/* returns 1 when inserted (was absent) */
static int kset_insert(KSet *s, uint64_t k) {
    if ((s->n + 1) * 2 > s->cap) kset_grow(s);
    uint32_t m = s->cap - 1, h = kmix(k) & m;
    while (s->keys[h] != UINT64_MAX) { if (s->keys[h] == k) return 0; h = (h + 1) & m; }
    s->keys[h] = k; s->n++;
    return 1;
}
static void kset_grow(KSet *s) {
    KSet t; t.cap = s->cap * 2; t.n = 0;
    t.keys = (uint64_t *)malloc(sizeof(uint64_t) * t.cap);
    memset(t.keys, 0xff, sizeof(uint64_t) * t.cap);
    for (uint32_t i = 0; i < s->cap; i++) if (s->keys[i] != UINT64_MAX) kset_insert(&t, s->keys[i]);
    free(s->keys); *s = t;
}
static inline uint64_t ekey(uint32_t a, uint32_t b) {
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ((uint64_t)lo << 32) | hi;
}

typedef struct { uint32_t *d; size_t n, cap; } UVec;
static void uv_push(UVec *v, uint32_t x) {
    if (v->n == v->cap) { v->cap = v->cap ? v->cap * 2 : 8; v->d = (uint32_t *)realloc(v->d, v->cap * 4); }
    v->d[v->n++] = x;
}
static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}
static size_t sort_dedup(uint32_t *a, size_t n) {
    if (!n) return 0;
    qsort(a, n, 4, cmp_u32);
    size_t m = 1;
    for (size_t i = 1; i < n; i++) if (a[i] != a[m - 1]) a[m++] = a[i];
    return m;
}
static int contains_u32(const uint32_t *a, size_t n, uint32_t x) {
    for (size_t i = 0; i < n; i++) if (a[i] == x) return 1;
    return 0;
}

/* ------------------------------------------------------------------ */
/* data                                                                */
/* ------------------------------------------------------------------ */
typedef struct { uint32_t v0, v1; float rest, tc, cc; uint32_t type; } ODist;
typedef struct { uint32_t v0, v1, v2, v3; float rest, comp, pad0, pad1; } OBend;
/* GpuSewingConstraint (mesh.rs:904-933) */
typedef struct { uint32_t v0, v1; float cur, target, speed, comp, lock; } OSew;
typedef struct { uint32_t type; float fric, rest; v3 a; float r; v3 b; } OCol;
typedef struct { v3 p0; float fric; v3 p1; float thick; v3 p2; float rest; uint32_t flags; } OTri;
typedef struct { uint32_t v; float w; v3 target; } OPin;
/* GpuColliderEdge (mesh.rs:91-100) */
typedef struct { v3 p0; float th; v3 p1; float fr; v3 nrm; uint32_t flags; } OCEdge;

/* accumulator slots, SelfCollisionAccum (shaders/self_collision.wgsl:31-48) */
enum { A_DX, A_DY, A_DZ, A_CNT, A_PDX, A_PDY, A_PDZ, A_PCNT, A_CPX, A_CPY, A_CPZ, A_CNX, A_CNY,
       A_CNZ, A_UT, A_EEC, A_N };

struct OSim {
    int n;
    v3 *x, *p, *v;
    float *w, *orig_w, *thick;
    uint32_t *layer;
    v3 *x0; float *w0; /* initial vertices, simulation/mod.rs:376 */
    /* constraints */
    ODist *dist; int nd; uint32_t *dc_off, *dc_cnt; int ndc; float *dlam;
    OBend *bend; int nb; uint32_t *bc_off, *bc_cnt; int nbc; float *blam;
    OSew *sew; int nsw; uint32_t *sc_off, *sc_cnt; int nsc; float *slam;
    uint32_t *rep; /* sewing group of each vertex (its smallest member) */
    float sew_stiffness, sew_speed, sew_lock_dist; int sew_lock; /* mod.rs:637-640 */
    /* topology */
    uint32_t *adj_off, *adj_idx;
    uint32_t *th_off, *th_idx; float *th_rest;
    float *local_len;
    uint32_t *star_off, *star_idx; /* pairs */
    uint32_t *edges; uint32_t *ebits; int ne;
    uint32_t *island;
    float mean_edge, max_edge;
    int num_virtual;
    /* params */
    v3 g; float damping; float td, cd, sd, bd;
    int iters;
    int self_collision;
    float relief; int enable_relief; float max_disp_ratio; int exclude_neighbors; int untangle_opt;
    int max_search; int multi_layer;
    float cell; uint32_t table;
    int coupled, auto_coupled;
    float last_max_disp, last_eff_disp;
    float cloth_thickness;
    int single_sided_recovery;
    int sc_interval, ee_interval; /* self-collision / E-E substep intervals (dispatch.rs:105-114) */
    /* narrow-phase pair record of the latest self-collision pass (ocl_set_pair_recording) */
    int rec;
    uint32_t *rec_vt, *rec_ee;
    size_t rec_vt_n, rec_vt_cap, rec_ee_n, rec_ee_cap;
    /* bone SDF colliders (collision.wgsl:116-265) */
    uint32_t *atlas; uint32_t aw, ah, ad; int nbones;
    float *binfo;   /* nbones x 20 */
    float *bxf;     /* nbones x 32: world, inverse world (column-major) */
    /* colliders */
    OCol *cols; int ncols;
    OTri *tris; float *bounds; int ntris;
    /* edge colliders (edge_collision.wgsl), off by default (mod.rs:628-630) */
    int edge_collision; float emscale, emoff;
    OCEdge *ce; int nce; uint32_t *ce_cs, *ce_srt; float ce_cell;
    OPin *pins; int npins;
    /* self-collision scratch */
    int32_t *acc;  /* n * A_N */
    v3 *nrm;
    uint32_t *cs, *srt, *ecs, *esrt;
    /* contact-pair cache (self-collision algorithm 1), off by default
     * (simulation/mod.rs:582-600) */
    int pair_cache, pair_fallback, pair_margin_mode;
    uint32_t pair_qvt, pair_qee, pair_max_vt, pair_max_ee;
    float pair_safety, pair_hscale, pair_maxh;
    uint32_t *pvt, *pee; /* n * 8 slots of four vertex ids */
    uint32_t pcnt[4];
};
/* quota_for_budget, simulation/mod.rs:36-41 (PAIR_QUOTA_MAX = 8) */
static uint32_t quota_for_budget(uint32_t budget, uint32_t nv) {
    if (nv == 0) return 1u;
    uint32_t q = budget / nv;
    return q < 1u ? 1u : (q > 8u ? 8u : q);
}

/* ------------------------------------------------------------------ */
/* Welsh-Powell colouring, crates/cloth_core/src/coloring.rs:6-173       */
/* ------------------------------------------------------------------ */
typedef struct { int deg; int idx; } DegIdx;
static int cmp_degidx(const void *a, const void *b) {
    const DegIdx *x = (const DegIdx *)a, *y = (const DegIdx *)b;
    if (x->deg != y->deg) return x->deg > y->deg ? -1 : 1; /* Reverse(deg) */
    return (x->idx > y->idx) - (x->idx < y->idx);
}

/* Generic greedy colouring: verts_of(i) gives the constraint's conflict
 * vertex list (as registered in vertex_to_constraints), deg(i) the sort key.
 * Returns number of colours; colors[i] filled. */
static int wp_color(int nv, int nc, const uint32_t *vlist, const int *vcount, int stride,
                    const uint32_t *reg, const int *regcount, uint32_t *colors) {
    /* vertex_to_constraints built from reg lists in constraint order */
    int *cnt = (int *)calloc((size_t)nv + 1, sizeof(int));
    for (int i = 0; i < nc; i++)
        for (int k = 0; k < regcount[i]; k++) cnt[reg[i * stride + k] + 1]++;
    for (int v = 0; v < nv; v++) cnt[v + 1] += cnt[v];
    int *fill = (int *)malloc(sizeof(int) * ((size_t)nv + 1));
    memcpy(fill, cnt, sizeof(int) * ((size_t)nv + 1));
    int *v2c = (int *)malloc(sizeof(int) * ((size_t)cnt[nv] + 1));
    for (int i = 0; i < nc; i++)
        for (int k = 0; k < regcount[i]; k++) v2c[fill[reg[i * stride + k]]++] = i;
    DegIdx *ord = (DegIdx *)malloc(sizeof(DegIdx) * ((size_t)nc + 1));
    for (int i = 0; i < nc; i++) {
        int d = 0;
        for (int k = 0; k < vcount[i]; k++) {
            uint32_t v = vlist[i * stride + k];
            if ((int)v < nv) d += cnt[v + 1] - cnt[v];
        }
        ord[i].deg = d; ord[i].idx = i;
    }
    qsort(ord, (size_t)nc, sizeof(DegIdx), cmp_degidx);
    for (int i = 0; i < nc; i++) colors[i] = UINT32_MAX;
    int ncol = 0;
    int mark_cap = 64;
    int *mark = (int *)calloc((size_t)mark_cap, sizeof(int));
    int stamp = 0;
    for (int oi = 0; oi < nc; oi++) {
        int i = ord[oi].idx;
        stamp++;
        for (int k = 0; k < vcount[i]; k++) {
            uint32_t v = vlist[i * stride + k];
            if ((int)v >= nv) continue;
            for (int q = cnt[v]; q < cnt[v + 1]; q++) {
                int a = v2c[q];
                if (a != i && colors[a] != UINT32_MAX) {
                    int c = (int)colors[a];
                    if (c >= mark_cap) {
                        int nc2 = mark_cap;
                        while (nc2 <= c) nc2 *= 2;
                        mark = (int *)realloc(mark, sizeof(int) * (size_t)nc2);
                        memset(mark + mark_cap, 0, sizeof(int) * (size_t)(nc2 - mark_cap));
                        mark_cap = nc2;
                    }
                    mark[c] = stamp;
                }
            }
        }
        int c = 0;
        while (c < mark_cap && mark[c] == stamp) c++;
        colors[i] = (uint32_t)c;
        if (c >= ncol) ncol = c + 1;
    }
    free(mark); free(ord); free(v2c); free(fill); free(cnt);
    return ncol;
}

/* reorder into colour buckets (stable by original index), offsets/counts */
static void bucket_reorder(int nc, int ncol, const uint32_t *colors, uint32_t **off, uint32_t **cnt,
                           int *perm /* perm[sorted] = orig */) {
    *off = (uint32_t *)calloc((size_t)ncol + 1, 4);
    *cnt = (uint32_t *)calloc((size_t)ncol + 1, 4);
    for (int i = 0; i < nc; i++) (*cnt)[colors[i]]++;
    uint32_t acc = 0;
    for (int c = 0; c < ncol; c++) { (*off)[c] = acc; acc += (*cnt)[c]; }
    uint32_t *fill = (uint32_t *)malloc(4 * ((size_t)ncol + 1));
    memcpy(fill, *off, 4 * (size_t)ncol);
    for (int i = 0; i < nc; i++) perm[fill[colors[i]]++] = i;
    free(fill);
}

/* ------------------------------------------------------------------ */
/* Morton code, crates/cloth_core/src/mesh.rs:323-338                   */
/* ------------------------------------------------------------------ */
static uint32_t expand_bits_10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static uint32_t f2u_sat(float f) { /* Rust `as u32`: saturating, NaN -> 0 */
    if (!(f > 0.0f)) return 0;
    if (f >= 4294967295.0f) return UINT32_MAX;
    return (uint32_t)f;
}
static uint32_t morton3(v3 p, v3 bmin, v3 inv) {
    uint32_t x = f2u_sat(clampf((p.x - bmin.x) * inv.x, 0.0f, 1.0f) * 1023.0f);
    uint32_t y = f2u_sat(clampf((p.y - bmin.y) * inv.y, 0.0f, 1.0f) * 1023.0f);
    uint32_t z = f2u_sat(clampf((p.z - bmin.z) * inv.z, 0.0f, 1.0f) * 1023.0f);
    return (expand_bits_10(x) << 2) | (expand_bits_10(y) << 1) | expand_bits_10(z);
}
typedef struct { uint32_t key; uint32_t idx; } KeyIdx;
static int cmp_keyidx(const void *a, const void *b) { /* stable by idx */
    const KeyIdx *x = (const KeyIdx *)a, *y = (const KeyIdx *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return (x->idx > y->idx) - (x->idx < y->idx);
}

/* entry of edge -> opposite vertex map (mesh.rs:508-522 / :655-669) */
typedef struct { uint64_t key; uint32_t opp; uint32_t ord; } EOpp;
static int cmp_eopp(const void *a, const void *b) {
    const EOpp *x = (const EOpp *)a, *y = (const EOpp *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return (x->ord > y->ord) - (x->ord < y->ord);
}

static float dist3(const float *a, const float *b) { /* dx = a - b */
    float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return sqrtf(dx * dx + dy * dy + dz * dz);
}

static float stiff_to_compliance(float k) {
    if (k >= 5000.0f) return 0.0f;
    if (k > 0.0f) return 1.0f / k;
    return 1e10f;
}

/* ------------------------------------------------------------------ */
/* construction                                                        */
/* ------------------------------------------------------------------ */
/* unfolding about a seam edge e0->e1 (mesh.rs:795-809, :1436-1454): the
 * position of p along the edge and its distance from the edge line */
static int seam_frame(const float *e0, const float *e1, const float *p, float *sa, float *ha) {
    float ev[3] = {e1[0] - e0[0], e1[1] - e0[1], e1[2] - e0[2]};
    float len = sqrtf(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]);
    if (len <= 1e-6f) return 0;
    float u[3] = {ev[0] / len, ev[1] / len, ev[2] / len};
    float d[3] = {p[0] - e0[0], p[1] - e0[1], p[2] - e0[2]};
    float sv = d[0] * u[0] + d[1] * u[1] + d[2] * u[2];
    float q[3] = {d[0] - sv * u[0], d[1] - sv * u[1], d[2] - sv * u[2]};
    *sa = sv;
    *ha = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    return 1;
}
static float seam_flat(float sa, float ha, float sb, float hb) {
    float ds = sa - sb, dh = ha + hb;
    return sqrtf(ds * ds + dh * dh);
}
/* compute_seam_two_hop_rest_length, mesh.rs:1382-1488 (oadj: the input
 * mesh's adjacency, sorted) */
static float seam_two_hop(int i, int nbr, const float *pos, const UVec *oadj, const uint32_t *rep) {
    uint32_t ri = rep[i], rn = rep[nbr];
    float best = FLT_MAX;
    for (size_t a = 0; a < oadj[i].n; a++) {
        uint32_t m1 = oadj[i].d[a], rm1 = rep[m1];
        if (rm1 == ri || rm1 == rn) continue;
        for (size_t b = 0; b < oadj[nbr].n; b++) {
            uint32_t m2 = oadj[nbr].d[b];
            if (rep[m2] != rm1) continue;
            if (m1 == m2) { /* case 5a */
                float d = dist3(pos + 3 * i, pos + 3 * nbr);
                if (d < best) best = d;
                continue;
            }
            int found = 0; /* case 5b: a seam edge from m1 and from m2 into one group */
            for (size_t c = 0; c < oadj[m1].n; c++) {
                uint32_t k1 = oadj[m1].d[c], rk1 = rep[k1];
                if (rk1 == rm1) continue;
                for (size_t e = 0; e < oadj[m2].n; e++) {
                    uint32_t k2 = oadj[m2].d[e];
                    if (rep[k2] != rk1) continue;
                    float sa, ha, sb, hb;
                    if (!seam_frame(pos + 3 * m1, pos + 3 * k1, pos + 3 * i, &sa, &ha)) continue;
                    if (!seam_frame(pos + 3 * m2, pos + 3 * k2, pos + 3 * nbr, &sb, &hb)) continue;
                    float fl = seam_flat(sa, ha, sb, hb);
                    if (fl < best) { best = fl; found = 1; }
                }
            }
            if (!found) { /* case 5c */
                float sl = dist3(pos + 3 * i, pos + 3 * m1) + dist3(pos + 3 * nbr, pos + 3 * m2);
                if (sl < best) best = sl;
            }
        }
    }
    return (best < FLT_MAX && isfinite(best) && best > 1e-5f) ? best : 0.0f;
}

typedef struct { uint64_t key; uint32_t a, b, opp, ord; } OSeam;
static int cmp_seam(const void *x, const void *y) {
    const OSeam *p = (const OSeam *)x, *q = (const OSeam *)y;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    return (p->ord > q->ord) - (p->ord < q->ord);
}

OSim *ocl_create(const float *pos, int n, const uint32_t *edges, int ne_in, const uint32_t *faces,
                 int nf, const float *inv_masses, const uint32_t *layer_ids,
                 const float *thicknesses, uint32_t layer_id, float thickness, float tension_k,
                 float compression_k, float shear_k, float bending_k) {
    return ocl_create_sewn(pos, n, edges, ne_in, faces, nf, inv_masses, layer_ids, thicknesses, layer_id,
                           thickness, tension_k, compression_k, shear_k, bending_k, NULL, 0, 1.0f);
}
OSim *ocl_create_sewn(const float *pos, int n, const uint32_t *edges, int ne_in, const uint32_t *faces,
                      int nf, const float *inv_masses, const uint32_t *layer_ids,
                      const float *thicknesses, uint32_t layer_id, float thickness, float tension_k,
                      float compression_k, float shear_k, float bending_k, const uint32_t *sew, int nsew,
                      float shrink_speed) {
    OSim *s = (OSim *)calloc(1, sizeof(OSim));
    s->emscale = 1.0f;
    s->sew_stiffness = 10000.0f;
    s->sew_lock = 1;
    s->sew_lock_dist = 0.02f;
    s->sew_speed = fmaxf(shrink_speed, 0.0f);
    s->sc_interval = 1;
    s->ee_interval = 1;
    s->n = n;
    size_t N = (size_t)(n > 0 ? n : 1);
    s->x = (v3 *)calloc(N, sizeof(v3)); s->p = (v3 *)calloc(N, sizeof(v3));
    s->v = (v3 *)calloc(N, sizeof(v3)); s->w = (float *)calloc(N, 4);
    s->orig_w = (float *)calloc(N, 4); s->thick = (float *)calloc(N, 4);
    s->layer = (uint32_t *)calloc(N, 4);
    s->x0 = (v3 *)calloc(N, sizeof(v3)); s->w0 = (float *)calloc(N, 4);
    /* vertices, mesh.rs:430-443 */
    for (int i = 0; i < n; i++) {
        s->x[i] = V3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        s->p[i] = s->x[i];
        s->w[i] = inv_masses ? inv_masses[i] : 1.0f;
        s->layer[i] = layer_ids ? layer_ids[i] : layer_id;
        s->thick[i] = thicknesses ? thicknesses[i] : thickness;
    }
    int nfv = 0; /* valid faces */
    uint32_t *vf = (uint32_t *)malloc(sizeof(uint32_t) * 3 * ((size_t)nf + 1));
    for (int f = 0; f < nf; f++) {
        uint32_t a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
        if ((int)a < n && (int)b < n && (int)c < n) {
            vf[3 * nfv] = a; vf[3 * nfv + 1] = b; vf[3 * nfv + 2] = c; nfv++;
        }
    }

    /* 1. distance constraints, mesh.rs:444-560 */
    float tc = stiff_to_compliance(tension_k), cc = stiff_to_compliance(compression_k),
          shc = stiff_to_compliance(shear_k);
    int dcap = ne_in * 3 + nf * 3 + 16;
    ODist *dl = (ODist *)malloc(sizeof(ODist) * (size_t)dcap);
    int nd = 0;
    KSet orig; kset_init(&orig, (uint32_t)ne_in + 1);
    for (int e = 0; e < ne_in; e++) {
        uint32_t a = edges[2 * e], b = edges[2 * e + 1];
        if ((int)a < n && (int)b < n && a != b) {
            ODist d; d.v0 = a; d.v1 = b; d.rest = dist3(pos + 3 * a, pos + 3 * b);
            d.tc = tc; d.cc = cc; d.type = 0;
            dl[nd++] = d;
            kset_insert(&orig, ekey(a, b));
        }
    }
    /* edge -> opposite vertices (face order preserved) */
    EOpp *eo = (EOpp *)malloc(sizeof(EOpp) * (3 * (size_t)nfv + 1));
    int neo = 0;
    for (int f = 0; f < nfv; f++) {
        uint32_t f0 = vf[3 * f], f1 = vf[3 * f + 1], f2 = vf[3 * f + 2];
        eo[neo].key = ekey(f0, f1); eo[neo].opp = f2; eo[neo].ord = (uint32_t)neo; neo++;
        eo[neo].key = ekey(f1, f2); eo[neo].opp = f0; eo[neo].ord = (uint32_t)neo; neo++;
        eo[neo].key = ekey(f2, f0); eo[neo].opp = f1; eo[neo].ord = (uint32_t)neo; neo++;
    }
    qsort(eo, (size_t)neo, sizeof(EOpp), cmp_eopp);
    if (nf > 0) {
        KSet exist; kset_init(&exist, (uint32_t)(ne_in + neo) + 1);
        for (uint32_t i = 0; i < orig.cap; i++) if (orig.keys[i] != UINT64_MAX) kset_insert(&exist, orig.keys[i]);
        for (int i = 0; i < neo;) {
            int j = i;
            while (j < neo && eo[j].key == eo[i].key) j++;
            uint64_t key = eo[i].key;
            if (!kset_has(&orig, key) && j - i == 2) {
                uint32_t o0 = eo[i].opp, o1 = eo[i + 1].opp;
                uint32_t pairs[2][2] = {{(uint32_t)(key >> 32), (uint32_t)key},
                                        {o0 < o1 ? o0 : o1, o0 < o1 ? o1 : o0}};
                for (int q = 0; q < 2; q++) {
                    uint32_t a = pairs[q][0], b = pairs[q][1];
                    if (a != b && kset_insert(&exist, ((uint64_t)a << 32) | b)) {
                        if (nd == dcap) { dcap *= 2; dl = (ODist *)realloc(dl, sizeof(ODist) * (size_t)dcap); }
                        ODist d; d.v0 = a; d.v1 = b; d.rest = dist3(pos + 3 * a, pos + 3 * b);
                        d.tc = shc; d.cc = shc; d.type = 1;
                        dl[nd++] = d;
                    }
                }
            }
            i = j;
        }
        kset_free(&exist);
    }
    /* colouring of distance constraints, coloring.rs:6-79 */
    s->nd = nd;
    {
        uint32_t *vl = (uint32_t *)malloc(sizeof(uint32_t) * 2 * ((size_t)nd + 1));
        int *vc = (int *)malloc(sizeof(int) * ((size_t)nd + 1));
        for (int i = 0; i < nd; i++) { vl[2 * i] = dl[i].v0; vl[2 * i + 1] = dl[i].v1; vc[i] = 2; }
        uint32_t *col = (uint32_t *)malloc(4 * ((size_t)nd + 1));
        int ncol = nd ? wp_color(n, nd, vl, vc, 2, vl, vc, col) : 0;
        int *perm = (int *)malloc(sizeof(int) * ((size_t)nd + 1));
        bucket_reorder(nd, ncol, col, &s->dc_off, &s->dc_cnt, perm);
        s->ndc = ncol;
        s->dist = (ODist *)malloc(sizeof(ODist) * ((size_t)nd + 1));
        for (int i = 0; i < nd; i++) s->dist[i] = dl[perm[i]];
        s->dlam = (float *)calloc((size_t)nd + 1, 4);
        free(vl); free(vc); free(col); free(perm);
    }
    /* 2. bending, mesh.rs:632-704 (+ 1D strand bending :840-905) */
    float bcomp = bending_k > 0.0f ? 1.0f / bending_k : 1e10f;
    int bcap = neo + ne_in + 16;
    OBend *bl = (OBend *)malloc(sizeof(OBend) * (size_t)bcap);
    int nb = 0;
    if (nf > 0) {
        for (int i = 0; i < neo;) {
            int j = i;
            while (j < neo && eo[j].key == eo[i].key) j++;
            if (kset_has(&orig, eo[i].key) && j - i == 2 && eo[i].opp != eo[i + 1].opp) {
                OBend b; b.v0 = (uint32_t)(eo[i].key >> 32); b.v1 = (uint32_t)eo[i].key;
                b.v2 = eo[i].opp; b.v3 = eo[i + 1].opp;
                b.rest = dist3(pos + 3 * b.v2, pos + 3 * b.v3);
                b.comp = bcomp; b.pad0 = 0.0f; b.pad1 = 0.0f;
                bl[nb++] = b;
            }
            i = j;
        }
    }
    /* sewing groups (mesh.rs:706-737): union-find, union into the smaller root */
    uint32_t *rep = (uint32_t *)malloc(4 * N);
    uint8_t *has_sew = (uint8_t *)calloc(N, 1);
    for (int i = 0; i < n; i++) rep[i] = (uint32_t)i;
    for (int k = 0; k < nsew; k++) {
        uint32_t u = sew[2 * k], v = sew[2 * k + 1];
        if ((int)u < n && (int)v < n && u != v) {
            has_sew[u] = has_sew[v] = 1;
            uint32_t ru = u, rv = v;
            while (ru != rep[ru]) ru = rep[ru];
            while (rv != rep[rv]) rv = rep[rv];
            if (ru != rv) { if (ru < rv) rep[rv] = ru; else rep[ru] = rv; }
        }
    }
    for (int i = 0; i < n; i++) { uint32_t r = (uint32_t)i; while (r != rep[r]) r = rep[r]; rep[i] = r; }
    s->rep = rep;
    /* seam-gated bending, mesh.rs:740-838: single-triangle edges whose ends
     * are both sewn into two different groups, paired per group pair */
    if (nsew > 0 && nf > 0) {
        OSeam *se = (OSeam *)malloc(sizeof(OSeam) * ((size_t)neo + 1));
        int nse = 0;
        for (int i = 0; i < neo;) {
            int j = i;
            while (j < neo && eo[j].key == eo[i].key) j++;
            uint32_t ea = (uint32_t)(eo[i].key >> 32), eb = (uint32_t)eo[i].key;
            if (j - i == 1 && has_sew[ea] && has_sew[eb] && rep[ea] != rep[eb]) {
                OSeam q;
                q.key = ekey(rep[ea], rep[eb]);
                q.a = rep[ea] < rep[eb] ? ea : eb; q.b = rep[ea] < rep[eb] ? eb : ea;
                q.opp = eo[i].opp; q.ord = (uint32_t)nse;
                se[nse++] = q;
            }
            i = j;
        }
        qsort(se, (size_t)nse, sizeof(OSeam), cmp_seam);
        for (int i = 0; i < nse;) {
            int j = i;
            while (j < nse && se[j].key == se[i].key) j++;
            if (j - i == 2) {
                OSeam A = se[i], B = se[i + 1];
                uint32_t v2 = A.opp, v3 = B.opp;
                float sa, ha, sb, hb;
                if (!(A.a == B.a || A.b == B.b || v2 == v3 || rep[v2] == rep[v3]) &&
                    seam_frame(pos + 3 * A.a, pos + 3 * A.b, pos + 3 * v2, &sa, &ha) &&
                    seam_frame(pos + 3 * B.a, pos + 3 * B.b, pos + 3 * v3, &sb, &hb)) {
                    float flat = seam_flat(sa, ha, sb, hb);
                    if (flat > 1e-5f) {
                        if (nb == bcap) { bcap *= 2; bl = (OBend *)realloc(bl, sizeof(OBend) * (size_t)bcap); }
                        OBend b; b.v0 = A.a; b.v1 = B.a; b.v2 = v2; b.v3 = v3; b.rest = flat; b.comp = bcomp;
                        b.pad0 = 1.0f; b.pad1 = fmaxf(flat * 0.5f, 0.01f);
                        bl[nb++] = b;
                    }
                }
            }
            i = j;
        }
        free(se);
    }
    {
        KSet fe; kset_init(&fe, (uint32_t)(3 * nf) + 1);
        for (int f = 0; f < nf; f++) {
            uint32_t f0 = faces[3 * f], f1 = faces[3 * f + 1], f2 = faces[3 * f + 2];
            kset_insert(&fe, ekey(f0, f1)); kset_insert(&fe, ekey(f1, f2)); kset_insert(&fe, ekey(f2, f0));
        }
        UVec *sadj = (UVec *)calloc(N, sizeof(UVec));
        int any = 0;
        for (int e = 0; e < ne_in; e++) {
            uint32_t a = edges[2 * e], b = edges[2 * e + 1];
            if ((int)a < n && (int)b < n && a != b && !kset_has(&fe, ekey(a, b))) {
                uv_push(&sadj[a], b); uv_push(&sadj[b], a); any = 1;
            }
        }
        if (any) {
            KSet bp; kset_init(&bp, (uint32_t)nb + 16);
            for (int i = 0; i < nb; i++) kset_insert(&bp, ekey(bl[i].v2, bl[i].v3));
            for (int u = 0; u < n; u++) {
                UVec *nbv = &sadj[u];
                if (nbv->n < 2) continue;
                for (size_t i = 0; i < nbv->n; i++)
                    for (size_t j = i + 1; j < nbv->n; j++) {
                        uint32_t a = nbv->d[i], b = nbv->d[j];
                        if (a != b && kset_insert(&bp, ekey(a, b))) {
                            if (nb == bcap) { bcap *= 2; bl = (OBend *)realloc(bl, sizeof(OBend) * (size_t)bcap); }
                            OBend c; c.v0 = (uint32_t)u; c.v1 = (uint32_t)u; c.v2 = a; c.v3 = b;
                            c.rest = dist3(pos + 3 * a, pos + 3 * b);
                            c.comp = fmaxf(bcomp * 10.0f, 0.5f); c.pad0 = 2.0f; c.pad1 = 0.0f;
                            bl[nb++] = c;
                        }
                    }
            }
            kset_free(&bp);
        }
        for (int i = 0; i < n; i++) free(sadj[i].d);
        free(sadj);
        kset_free(&fe);
    }
    /* colouring of bending constraints, coloring.rs:82-173 */
    s->nb = nb;
    {
        uint32_t *vl = (uint32_t *)malloc(sizeof(uint32_t) * 4 * ((size_t)nb + 1));
        int *vc = (int *)malloc(sizeof(int) * ((size_t)nb + 1));
        uint32_t *rg = (uint32_t *)malloc(sizeof(uint32_t) * 4 * ((size_t)nb + 1));
        int *rc = (int *)malloc(sizeof(int) * ((size_t)nb + 1));
        for (int i = 0; i < nb; i++) {
            OBend *c = &bl[i];
            int k = 0;
            rg[4 * i + k++] = c->v2; rg[4 * i + k++] = c->v3;
            if (c->pad0 > 0.5f) {
                if ((int)c->v0 < n && c->v0 != c->v2 && c->v0 != c->v3) rg[4 * i + k++] = c->v0;
                if ((int)c->v1 < n && c->v1 != c->v2 && c->v1 != c->v3 && c->v1 != c->v0) rg[4 * i + k++] = c->v1;
                vl[4 * i] = c->v2; vl[4 * i + 1] = c->v3; vl[4 * i + 2] = c->v0; vl[4 * i + 3] = c->v1;
                vc[i] = 4;
            } else {
                vl[4 * i] = c->v2; vl[4 * i + 1] = c->v3; vc[i] = 2;
            }
            rc[i] = k;
        }
        /* for seam/strand entries the degree sums v2,v3,v0,v1 and the used-colour
         * scan visits v0,v1,v2,v3 (both orders give the same result) */
        uint32_t *col = (uint32_t *)malloc(4 * ((size_t)nb + 1));
        int ncol = nb ? wp_color(n, nb, vl, vc, 4, rg, rc, col) : 0;
        int *perm = (int *)malloc(sizeof(int) * ((size_t)nb + 1));
        bucket_reorder(nb, ncol, col, &s->bc_off, &s->bc_cnt, perm);
        s->nbc = ncol;
        s->bend = (OBend *)malloc(sizeof(OBend) * ((size_t)nb + 1));
        for (int i = 0; i < nb; i++) s->bend[i] = bl[perm[i]];
        s->blam = (float *)calloc((size_t)nb + 1, 4);
        free(vl); free(vc); free(rg); free(rc); free(col); free(perm);
    }
    free(bl);
    /* 3. sewing constraints, mesh.rs:904-936; colouring coloring.rs:236-300 */
    {
        s->sew = (OSew *)malloc(sizeof(OSew) * ((size_t)nsew + 1));
        OSew *sl = (OSew *)malloc(sizeof(OSew) * ((size_t)nsew + 1));
        int ns = 0;
        for (int k = 0; k < nsew; k++) {
            uint32_t a = sew[2 * k], b = sew[2 * k + 1];
            if ((int)a < n && (int)b < n && a != b) {
                OSew c; c.v0 = a; c.v1 = b; c.cur = dist3(pos + 3 * a, pos + 3 * b); c.target = 0.0f;
                c.speed = fmaxf(shrink_speed, 0.0f); c.comp = 0.0f; c.lock = 1.0f; /* stiffness 10000, lock on */
                sl[ns++] = c;
            }
        }
        uint32_t *vl = (uint32_t *)malloc(4 * (2 * (size_t)ns + 1));
        int *vc = (int *)malloc(sizeof(int) * ((size_t)ns + 1));
        for (int i = 0; i < ns; i++) { vl[2 * i] = sl[i].v0; vl[2 * i + 1] = sl[i].v1; vc[i] = 2; }
        uint32_t *col = (uint32_t *)malloc(4 * ((size_t)ns + 1));
        int ncol = ns ? wp_color(n, ns, vl, vc, 2, vl, vc, col) : 0;
        int *perm = (int *)malloc(sizeof(int) * ((size_t)ns + 1));
        bucket_reorder(ns, ncol, col, &s->sc_off, &s->sc_cnt, perm);
        for (int i = 0; i < ns; i++) s->sew[i] = sl[perm[i]];
        s->nsw = ns; s->nsc = ncol;
        s->slam = (float *)calloc((size_t)ns + 1, 4);
        free(sl); free(vl); free(vc); free(col); free(perm);
    }
    /* 4. adjacency + local edge lengths, mesh.rs:949-1090 */
    UVec *adj = (UVec *)calloc(N, sizeof(UVec));
    float *lsum = (float *)calloc(N, 4);
    uint32_t *lcnt = (uint32_t *)calloc(N, 4);
    float total = 0.0f, maxe = 0.0f; uint32_t valid = 0;
    for (int e = 0; e < ne_in; e++) {
        uint32_t a = edges[2 * e], b = edges[2 * e + 1];
        if ((int)a < n && (int)b < n && a != b) {
            float len = dist3(pos + 3 * a, pos + 3 * b);
            total += len;
            if (len > maxe) maxe = len;
            valid++;
            uv_push(&adj[a], b); uv_push(&adj[b], a);
            lsum[a] += len; lcnt[a]++; lsum[b] += len; lcnt[b]++;
        }
    }
    s->mean_edge = valid > 0 ? total / (float)valid : 0.0f;
    s->max_edge = maxe;
    s->local_len = (float *)malloc(4 * N);
    for (int i = 0; i < n; i++)
        s->local_len[i] = lcnt[i] > 0 ? lsum[i] / (float)lcnt[i] : fmaxf(thickness, 0.01f);
    for (int i = 0; i < n; i++) adj[i].n = sort_dedup(adj[i].d, adj[i].n);
    /* the input mesh's adjacency, kept for two-hop rest lengths */
    UVec *oadj = (UVec *)calloc(N, sizeof(UVec));
    for (int i = 0; i < n; i++)
        for (size_t k = 0; k < adj[i].n; k++) uv_push(&oadj[i], adj[i].d[k]);
    int sewn = 0;
    for (int i = 0; i < n; i++) if (rep[i] != (uint32_t)i) sewn = 1;
    if (sewn) { /* mesh.rs:1026-1058: group members adjacent to each other and to all their neighbours */
        for (int g = 0; g < n; g++) {
            if (rep[g] != (uint32_t)g) continue;
            UVec mem = {0}, sh = {0};
            for (int i = g; i < n; i++) if (rep[i] == (uint32_t)g) uv_push(&mem, (uint32_t)i);
            if (mem.n > 1) {
                for (size_t a = 0; a < mem.n; a++)
                    for (size_t b = 0; b < mem.n; b++)
                        if (a != b) uv_push(&adj[mem.d[a]], mem.d[b]);
                for (size_t a = 0; a < mem.n; a++)
                    for (size_t k = 0; k < oadj[mem.d[a]].n; k++) {
                        uint32_t w = oadj[mem.d[a]].d[k];
                        if (rep[w] != (uint32_t)g) uv_push(&sh, w);
                    }
                sh.n = sort_dedup(sh.d, sh.n);
                for (size_t a = 0; a < mem.n; a++)
                    for (size_t k = 0; k < sh.n; k++) { uv_push(&adj[mem.d[a]], sh.d[k]); uv_push(&adj[sh.d[k]], mem.d[a]); }
            }
            free(mem.d); free(sh.d);
        }
    }
    s->adj_off = (uint32_t *)malloc(4 * (N + 1));
    size_t tot_adj = 0;
    for (int i = 0; i < n; i++) { adj[i].n = sort_dedup(adj[i].d, adj[i].n); tot_adj += adj[i].n; }
    s->adj_idx = (uint32_t *)malloc(4 * (tot_adj + 1));
    {
        uint32_t o = 0;
        for (int i = 0; i < n; i++) {
            s->adj_off[i] = o;
            memcpy(s->adj_idx + o, adj[i].d, 4 * adj[i].n);
            o += (uint32_t)adj[i].n;
        }
        s->adj_off[n] = o;
    }
    /* 4b. two-hop CSR, mesh.rs:1092-1199: the hop sets from the sewing-
     * extended adjacency; true two-hop pairs exclude the same group and
     * pairs adjacent in the input or in the group-contracted mesh */
    UVec *chop = (UVec *)calloc(N, sizeof(UVec));
    for (int e = 0; e < ne_in; e++) {
        uint32_t a = edges[2 * e], b = edges[2 * e + 1];
        if ((int)a < n && (int)b < n && a != b && rep[a] != rep[b]) { uv_push(&chop[rep[a]], rep[b]); uv_push(&chop[rep[b]], rep[a]); }
    }
    for (int i = 0; i < n; i++) chop[i].n = sort_dedup(chop[i].d, chop[i].n);
    uint8_t *isface = (uint8_t *)calloc(N, 1);
    for (int f = 0; f < nf; f++)
        for (int k = 0; k < 3; k++) if ((int)faces[3 * f + k] < n) isface[faces[3 * f + k]] = 1;
    {
        UVec th = {0}, all = {0};
        float *rest = NULL; size_t rcap = 0, rn = 0;
        s->th_off = (uint32_t *)malloc(4 * (N + 1));
        uint32_t *tmp = NULL; size_t tcap = 0;
        for (int i = 0; i < n; i++) {
            size_t m = 1;
            for (uint32_t k = s->adj_off[i]; k < s->adj_off[i + 1]; k++) {
                uint32_t u = s->adj_idx[k];
                m += 1 + (s->adj_off[u + 1] - s->adj_off[u]);
            }
            if (m > tcap) { tcap = m * 2; tmp = (uint32_t *)realloc(tmp, 4 * tcap); }
            size_t q = 0;
            tmp[q++] = (uint32_t)i;
            for (uint32_t k = s->adj_off[i]; k < s->adj_off[i + 1]; k++) {
                uint32_t u = s->adj_idx[k];
                tmp[q++] = u;
                for (uint32_t ku = s->adj_off[u]; ku < s->adj_off[u + 1]; ku++) tmp[q++] = s->adj_idx[ku];
            }
            q = sort_dedup(tmp, q);
            s->th_off[i] = (uint32_t)th.n;
            for (size_t k = 0; k < q; k++) {
                uint32_t nbr = tmp[k];
                uv_push(&th, nbr);
                int true2 = nbr != (uint32_t)i && isface[i] && isface[nbr] && rep[i] != rep[nbr] &&
                            !contains_u32(oadj[i].d, oadj[i].n, nbr) &&
                            !contains_u32(chop[rep[i]].d, chop[rep[i]].n, rep[nbr]);
                float d = 0.0f;
                if (true2) {
                    /* within two hops of the input mesh: plain distance */
                    int orig2 = contains_u32(oadj[i].d, oadj[i].n, nbr);
                    for (size_t a = 0; a < oadj[i].n && !orig2; a++) {
                        uint32_t u = oadj[i].d[a];
                        orig2 = contains_u32(oadj[u].d, oadj[u].n, nbr);
                    }
                    d = orig2 ? dist3(pos + 3 * i, pos + 3 * nbr) : seam_two_hop(i, (int)nbr, pos, oadj, rep);
                }
                if (rn == rcap) { rcap = rcap ? rcap * 2 : 64; rest = (float *)realloc(rest, 4 * rcap); }
                rest[rn++] = d;
            }
        }
        s->th_off[n] = (uint32_t)th.n;
        s->th_idx = th.d ? th.d : (uint32_t *)malloc(4);
        s->th_rest = rest ? rest : (float *)malloc(4);
        free(tmp); (void)all;
    }
    /* 5. star pairs, mesh.rs:1201-1221 */
    {
        UVec *st = (UVec *)calloc(N, sizeof(UVec));
        for (int f = 0; f < nfv; f++) {
            uint32_t f0 = vf[3 * f], f1 = vf[3 * f + 1], f2 = vf[3 * f + 2];
            uv_push(&st[f0], f1); uv_push(&st[f0], f2);
            uv_push(&st[f1], f2); uv_push(&st[f1], f0);
            uv_push(&st[f2], f0); uv_push(&st[f2], f1);
        }
        size_t tot = 0;
        for (int i = 0; i < n; i++) tot += st[i].n;
        s->star_off = (uint32_t *)malloc(4 * (N + 1));
        s->star_idx = (uint32_t *)malloc(4 * (tot + 2));
        uint32_t o = 0;
        for (int i = 0; i < n; i++) {
            s->star_off[i] = o / 2;
            memcpy(s->star_idx + o, st[i].d, 4 * st[i].n);
            o += (uint32_t)st[i].n;
            free(st[i].d);
        }
        s->star_off[n] = o / 2;
        free(st);
    }
    /* 7. islands, mesh.rs:1233-1256 */
    s->island = (uint32_t *)malloc(4 * N);
    {
        for (int i = 0; i < n; i++) s->island[i] = UINT32_MAX;
        uint32_t *q = (uint32_t *)malloc(4 * N);
        uint32_t cur = 0;
        for (int i = 0; i < n; i++) {
            if (s->island[i] != UINT32_MAX) continue;
            size_t h = 0, t = 0;
            s->island[i] = cur; q[t++] = (uint32_t)i;
            while (h < t) {
                uint32_t u = q[h++];
                for (uint32_t k = s->adj_off[u]; k < s->adj_off[u + 1]; k++) {
                    uint32_t v = s->adj_idx[k];
                    if ((int)v < n && s->island[v] == UINT32_MAX) { s->island[v] = cur; q[t++] = v; }
                }
            }
            cur++;
        }
        free(q);
    }
    /* unique Morton-sorted edges, mesh.rs:1258-1289 */
    {
        uint32_t *ge = (uint32_t *)malloc(sizeof(uint32_t) * 2 * ((size_t)ne_in + 1));
        int ng = 0;
        KSet es; kset_init(&es, (uint32_t)ne_in + 1);
        for (int e = 0; e < ne_in; e++) {
            uint32_t a = edges[2 * e], b = edges[2 * e + 1];
            if ((int)a < n && (int)b < n && a != b && kset_insert(&es, ekey(a, b))) {
                ge[2 * ng] = a < b ? a : b; ge[2 * ng + 1] = a < b ? b : a; ng++;
            }
        }
        kset_free(&es);
        if (ng > 0 && n > 0) {
            v3 bmin = V3(3.4028235e38f, 3.4028235e38f, 3.4028235e38f), bmax = vneg(bmin);
            for (int i = 0; i < n; i++) {
                bmin.x = fminf(bmin.x, pos[3 * i]); bmin.y = fminf(bmin.y, pos[3 * i + 1]); bmin.z = fminf(bmin.z, pos[3 * i + 2]);
                bmax.x = fmaxf(bmax.x, pos[3 * i]); bmax.y = fmaxf(bmax.y, pos[3 * i + 1]); bmax.z = fmaxf(bmax.z, pos[3 * i + 2]);
            }
            v3 inv = V3(1.0f / fmaxf(bmax.x - bmin.x, 1e-5f), 1.0f / fmaxf(bmax.y - bmin.y, 1e-5f),
                        1.0f / fmaxf(bmax.z - bmin.z, 1e-5f));
            KeyIdx *ki = (KeyIdx *)malloc(sizeof(KeyIdx) * (size_t)ng);
            for (int e = 0; e < ng; e++) {
                const float *p0 = pos + 3 * ge[2 * e], *p1 = pos + 3 * ge[2 * e + 1];
                v3 mid = V3((p0[0] + p1[0]) * 0.5f, (p0[1] + p1[1]) * 0.5f, (p0[2] + p1[2]) * 0.5f);
                ki[e].key = morton3(mid, bmin, inv); ki[e].idx = (uint32_t)e;
            }
            qsort(ki, (size_t)ng, sizeof(KeyIdx), cmp_keyidx);
            uint32_t *g2 = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (size_t)ng);
            for (int e = 0; e < ng; e++) { g2[2 * e] = ge[2 * ki[e].idx]; g2[2 * e + 1] = ge[2 * ki[e].idx + 1]; }
            free(ge); ge = g2; free(ki);
        }
        s->edges = ge; s->ne = ng;
        /* 8. open-boundary bits, mesh.rs:1291-1344 */
        int nw = (ng + 31) / 32;
        s->ebits = (uint32_t *)calloc((size_t)nw + 1, 4);
        if (nf > 0) {
            /* raw triangle count per edge key */
            EOpp *rc = (EOpp *)malloc(sizeof(EOpp) * (3 * (size_t)nf + 1));
            int nrc = 0;
            for (int f = 0; f < nf; f++) {
                uint32_t f0 = faces[3 * f], f1 = faces[3 * f + 1], f2 = faces[3 * f + 2];
                uint32_t te[3][2] = {{f0, f1}, {f1, f2}, {f2, f0}};
                for (int k = 0; k < 3; k++) {
                    uint32_t a = te[k][0], b = te[k][1];
                    uint32_t ea = a < b ? a : b, eb = a < b ? b : a;
                    if ((int)ea < n && (int)eb < n && ea != eb) { rc[nrc].key = ekey(ea, eb); rc[nrc].ord = (uint32_t)nrc; rc[nrc].opp = 0; nrc++; }
                }
            }
            qsort(rc, (size_t)nrc, sizeof(EOpp), cmp_eopp);
            /* the same counts between sewing groups (contracted mesh) */
            EOpp *cc = (EOpp *)malloc(sizeof(EOpp) * ((size_t)nrc + 1));
            int ncc = 0;
            for (int q = 0; q < nrc; q++) {
                uint32_t a = rep[(uint32_t)(rc[q].key >> 32)], b = rep[(uint32_t)rc[q].key];
                if (a != b) { cc[ncc].key = ekey(a, b); cc[ncc].ord = (uint32_t)ncc; cc[ncc].opp = 0; ncc++; }
            }
            qsort(cc, (size_t)ncc, sizeof(EOpp), cmp_eopp);
            for (int e = 0; e < ng; e++) {
                uint32_t ra = rep[ge[2 * e]], rb = rep[ge[2 * e + 1]];
                if (ra == rb) continue;
                uint64_t k = ekey(ge[2 * e], ge[2 * e + 1]);
                /* binary search count */
                int lo = 0, hi = nrc;
                while (lo < hi) { int m = (lo + hi) / 2; if (rc[m].key < k) lo = m + 1; else hi = m; }
                int c = 0;
                while (lo + c < nrc && rc[lo + c].key == k) c++;
                int open = c == 0;
                if (c == 1) {
                    uint64_t kc = ekey(ra, rb);
                    lo = 0; hi = ncc;
                    while (lo < hi) { int m = (lo + hi) / 2; if (cc[m].key < kc) lo = m + 1; else hi = m; }
                    int c2 = 0;
                    while (lo + c2 < ncc && cc[lo + c2].key == kc) c2++;
                    open = c2 == 1;
                }
                if (open) s->ebits[e >> 5] |= 1u << (e & 31);
            }
            free(rc); free(cc);
        } else {
            for (int e = 0; e < ng; e++)
                if (rep[ge[2 * e]] != rep[ge[2 * e + 1]]) s->ebits[e >> 5] |= 1u << (e & 31);
        }
    }
    /* automatic layers by island mean Z, simulation/pipelines.rs:131-167 */
    if (n > 0) {
        uint32_t first = s->layer[0];
        int same = 1;
        for (int i = 0; i < n; i++) if (s->layer[i] != first) { same = 0; break; }
        if (same) {
            uint32_t maxi = 0;
            for (int i = 0; i < n; i++) if (s->island[i] > maxi) maxi = s->island[i];
            if (maxi > 0) {
                float *zs = (float *)calloc(maxi + 1, 4);
                uint32_t *zc = (uint32_t *)calloc(maxi + 1, 4);
                for (int i = 0; i < n; i++) { zs[s->island[i]] += s->x[i].z; zc[s->island[i]]++; }
                /* stable sort of islands by mean z */
                typedef struct { float m; uint32_t id; } IM;
                IM *im = (IM *)malloc(sizeof(IM) * (maxi + 1));
                for (uint32_t k = 0; k <= maxi; k++) {
                    float c = (float)(zc[k] > 1 ? zc[k] : 1);
                    im[k].m = zs[k] / c; im[k].id = k;
                }
                for (uint32_t a = 1; a <= maxi; a++) { /* insertion sort: stable */
                    IM t = im[a]; int b = (int)a - 1;
                    while (b >= 0 && im[b].m > t.m) { im[b + 1] = im[b]; b--; }
                    im[b + 1] = t;
                }
                uint32_t *i2l = (uint32_t *)malloc(4 * (maxi + 1));
                for (uint32_t r = 0; r <= maxi; r++) i2l[im[r].id] = r;
                for (int i = 0; i < n; i++) s->layer[i] = i2l[s->island[i]];
                free(i2l); free(im); free(zs); free(zc);
            }
        }
    }
    s->multi_layer = 0;
    for (int i = 0; i < n; i++) if (s->layer[i] != s->layer[0]) { s->multi_layer = 1; break; }

    /* virtual particle count (sizes the hash table), virtual_mesh.rs:75-190 */
    {
        long long M = 0;
        float dthick = n > 0 ? s->thick[0] : 0.003f;
        float spacing = dthick * 1.5f;
        if (!(spacing <= 1e-6f) && n > 0 && nfv > 0) {
            KSet fe; kset_init(&fe, (uint32_t)(3 * nfv) + 1);
            for (int f = 0; f < nfv; f++) {
                uint32_t a = vf[3 * f], b = vf[3 * f + 1], c = vf[3 * f + 2];
                kset_insert(&fe, ekey(a, b)); kset_insert(&fe, ekey(b, c)); kset_insert(&fe, ekey(c, a));
            }
            for (int i = 0; i < s->nd; i++) {
                uint32_t u = s->dist[i].v0, v = s->dist[i].v1;
                if (!kset_has(&fe, ekey(u, v))) continue;
                float len = dist3(pos + 3 * v, pos + 3 * u);
                uint32_t ke = f2u_sat(ceilf(len / spacing));
                if (ke > 16) ke = 16;
                if (ke > 1) M += ke - 1;
            }
            for (int f = 0; f < nfv; f++) {
                const float *pa = pos + 3 * vf[3 * f], *pb = pos + 3 * vf[3 * f + 1], *pc = pos + 3 * vf[3 * f + 2];
                float lmax = fmaxf(fmaxf(dist3(pb, pa), dist3(pc, pb)), dist3(pa, pc));
                uint32_t k = f2u_sat(ceilf(lmax / spacing));
                if (k > 16) k = 16;
                if (k >= 3) M += (long long)(k - 1) * (k - 2) / 2;
            }
            kset_free(&fe);
        }
        if (M > 150000) M = 150000;
        s->num_virtual = (int)M;
    }
    /* hash sizing, simulation/pipelines.rs:898-912 */
    {
        float th = n > 0 ? s->thick[0] : 0.005f;
        float eb = fminf(fmaxf(s->max_edge * 0.85f, s->mean_edge * 1.0f), 0.025f);
        s->cell = fmaxf(fmaxf(th * 4.0f, eb), 0.01f);
        uint32_t cap = (uint32_t)(n + s->num_virtual) * 4u;
        uint32_t t = 1;
        while (t < cap) t <<= 1;
        if (t < 1024) t = 1024;
        if (t > 65536) t = 65536;
        s->table = t;
    }
    /* defaults, simulation/mod.rs:607-697 */
    s->g = V3(0.0f, 0.0f, -9.81f);
    s->damping = 1.0f;
    s->iters = 2;
    s->self_collision = 1;
    s->relief = 0.2f; s->enable_relief = 1; s->max_disp_ratio = 0.2f;
    s->exclude_neighbors = 1; s->untangle_opt = 1; s->max_search = 256;
    s->auto_coupled = 1;
    s->cloth_thickness = 0.005f;
    s->single_sided_recovery = 1;
    for (int i = 0; i < n; i++) { s->orig_w[i] = s->w[i]; s->x0[i] = s->x[i]; s->w0[i] = s->w[i]; }
    s->acc = (int32_t *)calloc(N * A_N, 4);
    s->nrm = (v3 *)calloc(N, sizeof(v3));
    s->cs = (uint32_t *)calloc((size_t)s->table + 1, 4);
    s->srt = (uint32_t *)calloc(N, 4);
    s->ecs = (uint32_t *)calloc((size_t)s->table + 1, 4);
    s->esrt = (uint32_t *)calloc((size_t)s->ne + 1, 4);
    s->pair_fallback = 1; s->pair_margin_mode = 1;
    s->pair_safety = 0.005f; s->pair_hscale = 1.3f; s->pair_maxh = 0.02f;
    {
        uint32_t b = (uint32_t)n * 8u;
        b = b < 8192u ? 8192u : (b > 262144u ? 262144u : b);
        s->pair_max_vt = s->pair_max_ee = b;
        s->pair_qvt = s->pair_qee = quota_for_budget(b, (uint32_t)n);
    }
    s->pvt = (uint32_t *)malloc(N * 8 * 16);
    s->pee = (uint32_t *)malloc(N * 8 * 16);
    memset(s->pvt, 0xFF, N * 8 * 16);
    memset(s->pee, 0xFF, N * 8 * 16);
    for (int i = 0; i < n; i++) { free(adj[i].d); free(oadj[i].d); free(chop[i].d); }
    free(oadj); free(chop); free(has_sew);
    free(adj); free(lsum); free(lcnt); free(isface); free(eo); free(dl); free(vf);
    kset_free(&orig);
    return s;
}

void ocl_destroy(OSim *s) {
    if (!s) return;
    void *ptrs[] = {s->x, s->p, s->v, s->w, s->orig_w, s->thick, s->layer, s->x0, s->w0, s->dist,
                    s->dc_off, s->dc_cnt, s->dlam, s->bend, s->bc_off, s->bc_cnt, s->blam,
                    s->adj_off, s->adj_idx, s->th_off, s->th_idx, s->th_rest, s->local_len,
                    s->star_off, s->star_idx, s->edges, s->ebits, s->island, s->cols, s->tris,
                    s->bounds, s->pins, s->acc, s->nrm, s->cs, s->srt, s->ecs, s->esrt,
                    s->atlas, s->binfo, s->bxf, s->sew, s->sc_off, s->sc_cnt, s->slam, s->rep,
                    s->ce, s->ce_cs, s->ce_srt, s->pvt, s->pee, s->rec_vt, s->rec_ee};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    free(s);
}

/* ------------------------------------------------------------------ */
/* setters                                                             */
/* ------------------------------------------------------------------ */
void ocl_set_gravity(OSim *s, float gx, float gy, float gz) { s->g = V3(gx, gy, gz); }
void ocl_set_damping(OSim *s, float d) { s->damping = fmaxf(d, 0.0f); }
void ocl_set_damping_all(OSim *s, float t, float c, float sh, float b) {
    s->td = fmaxf(t, 0.0f); s->cd = fmaxf(c, 0.0f); s->sd = fmaxf(sh, 0.0f); s->bd = fmaxf(b, 0.0f);
}
void ocl_set_solver_iterations(OSim *s, int it) { s->iters = it < 1 ? 1 : it; }
void ocl_set_enable_self_collision(OSim *s, int on) { s->self_collision = on != 0; }
void ocl_set_coupled_collider(OSim *s, int on) { s->coupled = on != 0; }
/* set_collider_options (simulation/mod.rs set_collider_options): only the
 * single-sided recovery flag changes results; cluster culling and the sweep
 * margin select broadphase variants whose contacts are the same. */
void ocl_set_collider_options(OSim *s, int cluster, int recovery, float sweep) {
    (void)cluster; (void)sweep;
    s->single_sided_recovery = recovery != 0;
}
/* simulation/mod.rs:920-950 */
void ocl_set_self_collision_options(OSim *s, float relief, float max_disp_ratio, int exclude_neighbors,
                                    int untangle, int max_iter) {
    s->relief = relief; s->max_disp_ratio = max_disp_ratio;
    s->enable_relief = relief < 0.999f;
    s->exclude_neighbors = exclude_neighbors != 0; s->untangle_opt = untangle != 0;
    s->max_search = max_iter;
}
/* compliance set directly (no stiffness mapping) */
void ocl_set_compliance_all(OSim *s, float tension, float compression, float shear, float bending) {
    for (int i = 0; i < s->nd; i++) {
        if (s->dist[i].type == 1) { s->dist[i].tc = shear; s->dist[i].cc = shear; }
        else { s->dist[i].tc = tension; s->dist[i].cc = compression; }
    }
    for (int i = 0; i < s->nb; i++)
        s->bend[i].comp = s->bend[i].pad0 > 1.5f ? fmaxf(bending * 10.0f, 0.5f) : bending;
}
static void push_col(OSim *s, OCol c) {
    s->cols = (OCol *)realloc(s->cols, sizeof(OCol) * (size_t)(s->ncols + 1));
    s->cols[s->ncols++] = c;
}
void ocl_add_sphere(OSim *s, const float *c, float r, float fric, float rest) {
    OCol k; memset(&k, 0, sizeof k); k.type = 0; k.fric = fric; k.rest = rest;
    k.a = V3(c[0], c[1], c[2]); k.r = r; push_col(s, k);
}
void ocl_add_capsule(OSim *s, const float *a, const float *b, float r, float fric, float rest) {
    OCol k; memset(&k, 0, sizeof k); k.type = 1; k.fric = fric; k.rest = rest;
    k.a = V3(a[0], a[1], a[2]); k.b = V3(b[0], b[1], b[2]); k.r = r; push_col(s, k);
}
void ocl_add_plane(OSim *s, const float *pt, const float *nrm, float fric, float rest) {
    OCol k; memset(&k, 0, sizeof k); k.type = 2; k.fric = fric; k.rest = rest;
    k.a = V3(pt[0], pt[1], pt[2]); k.b = V3(nrm[0], nrm[1], nrm[2]); k.r = 0.0f; push_col(s, k);
}
/* cloth_py/src/lib.rs:2175-2234 and upload_colliders, simulation/mod.rs:2613-2670 */
/* extract_collider_edges (mesh.rs:1503-1565): an edge per distinct
 * endpoint pair (keyed by the endpoints' bits), oriented as in the first
 * triangle that has it; thickness max, friction averaged, normals summed in
 * triangle order, then normalised; flags = AND of the single-sided bits.
 * build_collider_edge_grid (spatial_hash.rs:463-528): every cell the edge
 * passes through at half-cell sampling, once per distinct bucket. */
static inline uint32_t hash3(int32_t cx, int32_t cy, int32_t cz, uint32_t table);
static inline void cell_of(v3 p, float cell, int32_t *c);
typedef struct { uint32_t key[6]; uint32_t ord; } OEKey;
static int cmp_ekey(const void *x, const void *y) {
    const OEKey *p = (const OEKey *)x, *q = (const OEKey *)y;
    for (int k = 0; k < 6; k++) if (p->key[k] != q->key[k]) return p->key[k] < q->key[k] ? -1 : 1;
    return (p->ord > q->ord) - (p->ord < q->ord);
}
static int32_t sat_i32f(float f) {
    if (!(f == f)) return 0;
    if (f <= -2147483648.0f) return INT32_MIN;
    if (f >= 2147483647.0f) return INT32_MAX;
    return (int32_t)f;
}
static void build_collider_edges(OSim *s) {
    free(s->ce); free(s->ce_cs); free(s->ce_srt);
    s->ce = NULL; s->ce_cs = NULL; s->ce_srt = NULL; s->nce = 0;
    s->ce_cell = s->cell;
    const uint32_t T = 32768u;
    s->ce_cs = (uint32_t *)calloc((size_t)T + 1, 4);
    s->ce_srt = (uint32_t *)malloc(4);
    int nt = s->ntris;
    if (nt <= 0) return;
    OEKey *ks = (OEKey *)malloc(sizeof(OEKey) * 3 * (size_t)nt);
    for (int t = 0; t < nt; t++)
        for (int k = 0; k < 3; k++) {
            v3 a = k == 0 ? s->tris[t].p0 : (k == 1 ? s->tris[t].p1 : s->tris[t].p2);
            v3 b = k == 0 ? s->tris[t].p1 : (k == 1 ? s->tris[t].p2 : s->tris[t].p0);
            uint32_t ab[3], bb[3];
            memcpy(ab, &a, 12); memcpy(bb, &b, 12);
            int a_first = ab[0] != bb[0] ? ab[0] < bb[0] : (ab[1] != bb[1] ? ab[1] < bb[1] : ab[2] < bb[2]);
            OEKey q;
            memcpy(q.key, a_first ? ab : bb, 12); memcpy(q.key + 3, a_first ? bb : ab, 12);
            q.ord = (uint32_t)(3 * t + k);
            ks[3 * t + k] = q;
        }
    qsort(ks, 3 * (size_t)nt, sizeof(OEKey), cmp_ekey);
    s->ce = (OCEdge *)malloc(sizeof(OCEdge) * 3 * (size_t)nt);
    int ne = 0;
    for (int i = 0; i < 3 * nt;) {
        int j = i;
        while (j < 3 * nt && memcmp(ks[j].key, ks[i].key, sizeof ks[i].key) == 0) j++;
        OCEdge e;
        for (int q = i; q < j; q++) {
            int t = (int)(ks[q].ord / 3), k = (int)(ks[q].ord % 3);
            OTri *o = &s->tris[t];
            v3 e1 = vsub(o->p1, o->p0), e2 = vsub(o->p2, o->p0);
            v3 cr = V3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x);
            float cl = sqrtf(cr.x * cr.x + cr.y * cr.y + cr.z * cr.z);
            v3 tn = cl > 1e-12f ? V3(cr.x / cl, cr.y / cl, cr.z / cl) : V3(0.0f, 0.0f, 0.0f);
            uint32_t single = o->flags & 1u;
            if (q == i) {
                e.p0 = k == 0 ? o->p0 : (k == 1 ? o->p1 : o->p2);
                e.p1 = k == 0 ? o->p1 : (k == 1 ? o->p2 : o->p0);
                e.th = o->thick; e.fr = o->fric; e.nrm = tn; e.flags = single;
            } else {
                e.th = fmaxf(e.th, o->thick);
                e.fr = (e.fr + o->fric) * 0.5f;
                e.nrm = V3(e.nrm.x + tn.x, e.nrm.y + tn.y, e.nrm.z + tn.z);
                e.flags &= single;
            }
        }
        float nl = sqrtf(e.nrm.x * e.nrm.x + e.nrm.y * e.nrm.y + e.nrm.z * e.nrm.z);
        e.nrm = nl > 1e-6f ? V3(e.nrm.x / nl, e.nrm.y / nl, e.nrm.z / nl) : V3(0.0f, 0.0f, 0.0f);
        s->ce[ne++] = e;
        i = j;
    }
    free(ks);
    s->nce = ne;
    float safe = fmaxf(s->ce_cell, 1e-4f), pitch = safe * 0.5f;
    UVec hb = {0}, eb = {0}; /* (bucket, edge) entries */
    uint32_t *hs = NULL; size_t hcap = 0;
    for (int ei = 0; ei < ne; ei++) {
        OCEdge *e = &s->ce[ei];
        float dx = e->p1.x - e->p0.x, dy = e->p1.y - e->p0.y, dz = e->p1.z - e->p0.z;
        float len = sqrtf(dx * dx + dy * dy + dz * dz);
        float sf = ceilf(len / pitch);
        size_t steps = (sf == sf && sf > 0.0f) ? (sf >= 4096.0f ? 4096 : (size_t)sf) : 0;
        if (steps < 1) steps = 1;
        if (steps > 4096) steps = 4096;
        if (steps + 1 > hcap) { hcap = 2 * (steps + 1); hs = (uint32_t *)realloc(hs, 4 * hcap); }
        for (size_t k = 0; k <= steps; k++) {
            float t = (float)k / (float)steps;
            float px = e->p0.x + dx * t, py = e->p0.y + dy * t, pz = e->p0.z + dz * t;
            hs[k] = hash3(sat_i32f(floorf(px / safe)), sat_i32f(floorf(py / safe)), sat_i32f(floorf(pz / safe)), T);
        }
        size_t nh = sort_dedup(hs, steps + 1);
        for (size_t k = 0; k < nh; k++) { uv_push(&hb, hs[k]); uv_push(&eb, (uint32_t)ei); }
    }
    free(hs);
    for (size_t k = 0; k < hb.n; k++) s->ce_cs[hb.d[k] + 1]++;
    for (uint32_t h = 0; h < T; h++) s->ce_cs[h + 1] += s->ce_cs[h];
    free(s->ce_srt);
    s->ce_srt = (uint32_t *)malloc(4 * (hb.n + 1));
    uint32_t *cur = (uint32_t *)malloc(4 * (size_t)T);
    memcpy(cur, s->ce_cs, 4 * (size_t)T);
    for (size_t k = 0; k < hb.n; k++) s->ce_srt[cur[hb.d[k]]++] = eb.d[k];
    free(cur); free(hb.d); free(eb.d);
}
/* closest points of two segments (edge_collision.wgsl:96-149) */
static float eseg_closest(v3 p0, v3 p1, v3 q0, v3 q1, float *s_out, float *t_out) {
    v3 d1 = vsub(p1, p0), d2 = vsub(q1, q0), r = vsub(p0, q0);
    float a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= 1e-12f && e <= 1e-12f) { *s_out = 0.0f; *t_out = 0.0f; return vlen(vsub(p0, q0)); }
    if (a <= 1e-12f) {
        t = clampf(f / e, 0.0f, 1.0f);
    } else {
        float c = vdot(d1, r);
        if (e <= 1e-12f) {
            s = clampf(-c / a, 0.0f, 1.0f);
        } else {
            float b = vdot(d1, d2);
            float denom = a * e - b * b;
            if (denom > a * e * 1e-7f) s = clampf((b * f - c * e) / denom, 0.0f, 1.0f);
            t = (b * s + f) / e;
            if (t < 0.0f) { t = 0.0f; s = clampf(-c / a, 0.0f, 1.0f); }
            else if (t > 1.0f) { t = 1.0f; s = clampf((b - c) / a, 0.0f, 1.0f); }
        }
    }
    *s_out = s; *t_out = t;
    return vlen(vsub(vadd(p0, vmul(d1, s)), vadd(q0, vmul(d2, t))));
}
static void add_pin(OSim *s, uint32_t v, v3 d);
static void k_apply(OSim *s);
/* shaders/edge_collision.wgsl:150-276, then the apply pass (dispatch.rs:254-283) */
static void k_edge_collision(OSim *s) {
    if (s->nce > 0) {
        for (int ei = 0; ei < s->ne; ei++) {
            uint32_t u0 = s->edges[2 * ei], u1 = s->edges[2 * ei + 1];
            float w0 = s->w[u0], w1 = s->w[u1];
            if (w0 + w1 <= EPS) continue;
            v3 p0 = s->p[u0], p1 = s->p[u1];
            v3 pmid = vmul(vadd(p0, p1), 0.5f);
            float cth = fmaxf(s->thick[u0], s->thick[u1]);
            int32_t cc[3]; cell_of(pmid, s->ce_cell, cc);
            v3 lo = vmin(p0, p1), hi = vmax(p0, p1);
            for (int dz = -1; dz <= 1; dz++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        uint32_t h = hash3(cc[0] + dx, cc[1] + dy, cc[2] + dz, 32768u);
                        for (uint32_t k = s->ce_cs[h]; k < s->ce_cs[h + 1]; k++) {
                            const OCEdge *ce = &s->ce[s->ce_srt[k]];
                            float tgt = (cth + ce->th) * s->emscale + s->emoff;
                            v3 clo = vmin(ce->p0, ce->p1), chi = vmax(ce->p0, ce->p1);
                            if (hi.x + tgt < clo.x || lo.x - tgt > chi.x || hi.y + tgt < clo.y || lo.y - tgt > chi.y ||
                                hi.z + tgt < clo.z || lo.z - tgt > chi.z)
                                continue;
                            float sp_, tp_;
                            float dist = eseg_closest(p0, p1, ce->p0, ce->p1, &sp_, &tp_);
                            if (!(dist < tgt)) continue;
                            v3 diff = vsub(vadd(p0, vmul(vsub(p1, p0), sp_)), vadd(ce->p0, vmul(vsub(ce->p1, ce->p0), tp_)));
                            int single = (ce->flags & 1u) != 0u;
                            int has_n = vdot(ce->nrm, ce->nrm) > 0.25f;
                            v3 nrm = V3(0.0f, 0.0f, 1.0f);
                            float pen = tgt - dist;
                            if (single && has_n) {
                                float sd = vdot(diff, ce->nrm);
                                if (sd >= 0.0f) { nrm = dist > EPS ? vdiv(diff, dist) : ce->nrm; pen = tgt - dist; }
                                else { nrm = ce->nrm; pen = fminf(tgt - sd, tgt * 2.0f); }
                            } else if (dist > EPS) {
                                nrm = vdiv(diff, dist);
                            } else {
                                v3 cr = vcross(vsub(p1, p0), vsub(ce->p1, ce->p0));
                                float cl = vlen(cr);
                                if (cl > EPS) nrm = vdiv(cr, cl);
                            }
                            v3 push = vmul(nrm, pen);
                            float ca = 1.0f - sp_, cb = sp_;
                            float den = ca * ca * w0 + cb * cb * w1;
                            if (den > EPS) {
                                float f0 = fminf((ca * w0) / den, 2.0f), f1 = fminf((cb * w1) / den, 2.0f);
                                if (w0 > 0.0f) add_pin(s, u0, vmul(push, f0));
                                if (w1 > 0.0f) add_pin(s, u1, vmul(push, f1));
                            }
                        }
                    }
        }
    }
    k_apply(s);
}

void ocl_set_edge_collision(OSim *s, int enable, float margin_scale, float margin_offset) {
    s->edge_collision = enable != 0;
    s->emscale = fmaxf(margin_scale, 1.0f);
    s->emoff = fmaxf(margin_offset, 0.0f);
}
int ocl_num_collider_edges(const OSim *s) { return s->nce; }

void ocl_set_mesh_triangles(OSim *s, const float *tris, int T, float fric, float thick, float rest,
                            int single_sided, const float *attrs) {
    free(s->tris); free(s->bounds);
    s->tris = (OTri *)malloc(sizeof(OTri) * ((size_t)T + 1));
    s->bounds = (float *)malloc(sizeof(float) * 4 * ((size_t)T + 1));
    s->ntris = T;
    for (int t = 0; t < T; t++) {
        const float *q = tris + 9 * t;
        OTri o;
        o.p0 = V3(q[0], q[1], q[2]); o.p1 = V3(q[3], q[4], q[5]); o.p2 = V3(q[6], q[7], q[8]);
        if (attrs) {
            o.fric = attrs[4 * t]; o.thick = attrs[4 * t + 1]; o.rest = attrs[4 * t + 2];
            o.flags = f2u_sat(roundf(attrs[4 * t + 3]));
        } else {
            o.fric = fric; o.thick = thick; o.rest = rest; o.flags = single_sided ? 1u : 0u;
        }
        s->tris[t] = o;
    }
    if (T <= 0) { build_collider_edges(s); return; }
    /* Morton sort of triangle centroids (stable) */
    v3 bmin = V3(3.4028235e38f, 3.4028235e38f, 3.4028235e38f), bmax = vneg(bmin);
    for (int t = 0; t < T; t++) {
        OTri *o = &s->tris[t];
        v3 c = V3((o->p0.x + o->p1.x + o->p2.x) / 3.0f, (o->p0.y + o->p1.y + o->p2.y) / 3.0f,
                  (o->p0.z + o->p1.z + o->p2.z) / 3.0f);
        bmin = vmin(bmin, c); bmax = vmax(bmax, c);
    }
    v3 inv = V3(1.0f / fmaxf(bmax.x - bmin.x, 1e-5f), 1.0f / fmaxf(bmax.y - bmin.y, 1e-5f),
                1.0f / fmaxf(bmax.z - bmin.z, 1e-5f));
    KeyIdx *ki = (KeyIdx *)malloc(sizeof(KeyIdx) * (size_t)T);
    for (int t = 0; t < T; t++) {
        OTri *o = &s->tris[t];
        v3 c = V3((o->p0.x + o->p1.x + o->p2.x) / 3.0f, (o->p0.y + o->p1.y + o->p2.y) / 3.0f,
                  (o->p0.z + o->p1.z + o->p2.z) / 3.0f);
        ki[t].key = morton3(c, bmin, inv); ki[t].idx = (uint32_t)t;
    }
    qsort(ki, (size_t)T, sizeof(KeyIdx), cmp_keyidx);
    OTri *sorted = (OTri *)malloc(sizeof(OTri) * (size_t)T);
    for (int t = 0; t < T; t++) sorted[t] = s->tris[ki[t].idx];
    free(s->tris); s->tris = sorted; free(ki);
    for (int t = 0; t < T; t++) {
        OTri *o = &s->tris[t];
        float cx = (o->p0.x + o->p1.x + o->p2.x) / 3.0f, cy = (o->p0.y + o->p1.y + o->p2.y) / 3.0f,
              cz = (o->p0.z + o->p1.z + o->p2.z) / 3.0f;
        float ax = o->p0.x - cx, ay = o->p0.y - cy, az = o->p0.z - cz;
        float bx = o->p1.x - cx, by = o->p1.y - cy, bz = o->p1.z - cz;
        float qx = o->p2.x - cx, qy = o->p2.y - cy, qz = o->p2.z - cz;
        float d0 = ax * ax + ay * ay + az * az, d1 = bx * bx + by * by + bz * bz, d2 = qx * qx + qy * qy + qz * qz;
        float r = sqrtf(fmaxf(fmaxf(d0, d1), d2)) + o->thick;
        s->bounds[4 * t] = cx; s->bounds[4 * t + 1] = cy; s->bounds[4 * t + 2] = cz; s->bounds[4 * t + 3] = r;
    }
    build_collider_edges(s);
}
void ocl_clear_colliders(OSim *s) {
    free(s->cols); s->cols = NULL; s->ncols = 0;
    free(s->tris); s->tris = NULL; free(s->bounds); s->bounds = NULL; s->ntris = 0;
    build_collider_edges(s);
}
/* simulation/mod.rs:2768-2791 */
void ocl_set_pin(OSim *s, uint32_t v, const float *target, float w) {
    if ((int)v >= s->n) return;
    int k;
    for (k = 0; k < s->npins; k++) if (s->pins[k].v == v) break;
    if (k == s->npins) { s->pins = (OPin *)realloc(s->pins, sizeof(OPin) * (size_t)(s->npins + 1)); s->npins++; }
    s->pins[k].v = v; s->pins[k].w = w; s->pins[k].target = V3(target[0], target[1], target[2]);
    float cw = (w == w && fabsf(w) != INFINITY) ? clampf(w, 0.0f, 1.0f) : 0.0f;
    s->w[v] = s->orig_w[v] * (1.0f - cw);
}
void ocl_clear_pins(OSim *s) {
    for (int k = 0; k < s->npins; k++) s->w[s->pins[k].v] = s->orig_w[s->pins[k].v];
    free(s->pins); s->pins = NULL; s->npins = 0;
}

/* ------------------------------------------------------------------ */
/* kernels                                                             */
/* ------------------------------------------------------------------ */
/* shaders/predict.wgsl:33-55 */
static void k_predict(OSim *s, float dt_sub) {
    float dt = fmaxf(dt_sub, 1e-8f);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; i++) {
        if (s->w[i] <= 0.0f) { s->v[i] = V3(0, 0, 0); s->p[i] = s->x[i]; }
        else {
            float sc = fmaxf(0.0f, 1.0f - s->damping * dt);
            v3 gdt = vmul(s->g, dt);
            s->v[i] = vadd(vmul(s->v[i], sc), gdt);
            s->p[i] = vadd(s->x[i], vmul(s->v[i], dt));
        }
    }
}
/* shaders/pin.wgsl:56-92 */
static void k_pin(OSim *s, float dt_sub) {
    for (int k = 0; k < s->npins; k++) {
        OPin *pn = &s->pins[k];
        uint32_t vi = pn->v;
        float w = clampf(pn->w, 0.0f, 1.0f);
        if (w <= 0.0f) continue;
        float im = s->w[vi];
        if (im <= 0.0f) { s->p[vi] = pn->target; continue; }
        v3 d = vsub(s->p[vi], pn->target);
        float dist = vlen(d);
        if (!(dist > EPS)) continue;
        v3 nn = vdiv(d, dist);
        float dt = fmaxf(dt_sub, 1e-8f);
        float comp = 1e-3f * (1.0f - w) / fmaxf(w, 1e-6f);
        float alpha = comp / (dt * dt);
        float corr = -dist / (im + alpha);
        s->p[vi] = vadd(s->p[vi], vmul(nn, im * corr));
    }
}
/* shaders/distance.wgsl:60-124 */
static void k_distance(OSim *s, int cidx, float dt_sub) {
    uint32_t off = s->dc_off[cidx], cnt = s->dc_cnt[cidx];
#pragma omp parallel for schedule(static) if (cnt > 4096)
    for (uint32_t q = 0; q < cnt; q++) {
        uint32_t ci = off + q;
        ODist *c = &s->dist[ci];
        float w0 = s->w[c->v0], w1 = s->w[c->v1];
        float ws = w0 + w1;
        if (ws <= EPS) continue;
        v3 p0 = s->p[c->v0], p1 = s->p[c->v1];
        v3 delta = vsub(p0, p1);
        float dist = vlen(delta);
        if (dist <= EPS) continue;
        float cv = dist - c->rest;
        float comp = cv >= 0.0f ? c->tc : c->cc;
        if (comp >= 1e9f) continue;
        v3 dir = vdiv(delta, dist);
        float dt = fmaxf(dt_sub, 1e-8f);
        float alpha = comp / (dt * dt);
        float damp = c->type == 1 ? s->sd : (cv >= 0.0f ? s->td : s->cd);
        float tau = damp * 1e-5f;
        float gamma = fminf(tau / dt, 1e4f);
        v3 rel = vsub(vsub(p0, s->x[c->v0]), vsub(p1, s->x[c->v1]));
        float vp = vdot(dir, rel);
        float lam = s->dlam[ci];
        float dl = (-cv - alpha * lam - gamma * vp) / ((1.0f + gamma) * ws + alpha);
        s->dlam[ci] = lam + dl;
        float a0 = w0 * dl, a1 = -w1 * dl;
        s->p[c->v0] = vadd(s->p[c->v0], vmul(dir, a0));
        s->p[c->v1] = vadd(s->p[c->v1], vmul(dir, a1));
    }
}
/* shaders/sewing_shrink.wgsl:38-49 */
static void k_sew_shrink(OSim *s, float dt_sub) {
    float dt = fmaxf(dt_sub, 1e-8f);
    for (int i = 0; i < s->nsw; i++) s->sew[i].cur = fmaxf(s->sew[i].target, s->sew[i].cur - s->sew_speed * dt);
}
/* shaders/sewing.wgsl:57-110, settings from SimParams (dispatch.rs:29-35) */
static void k_sewing(OSim *s, int cidx, float dt_sub) {
    float scomp = s->sew_stiffness >= 5000.0f ? 0.0f : 1.0f / fmaxf(s->sew_stiffness, 1.0f);
    uint32_t off = s->sc_off[cidx], cnt = s->sc_cnt[cidx];
    for (uint32_t q = 0; q < cnt; q++) {
        uint32_t ci = off + q;
        OSew *c = &s->sew[ci];
        float w0 = s->w[c->v0], w1 = s->w[c->v1];
        float ws = w0 + w1;
        if (ws <= EPS) continue;
        v3 p0 = s->p[c->v0], p1 = s->p[c->v1];
        v3 delta = vsub(p0, p1);
        float dist = vlen(delta);
        if (dist <= EPS) continue;
        float dt = fmaxf(dt_sub, 1e-8f);
        v3 dir = vdiv(delta, dist);
        float target = c->cur, comp = scomp;
        float lock_thresh = fmaxf(s->thick[c->v0] + s->thick[c->v1], s->sew_lock_dist);
        if (s->sew_lock && dist <= lock_thresh) {
            comp = 0.0f;
            target = c->target;
            c->cur = c->target;
        }
        float alpha = comp / (dt * dt);
        float cv = dist - target;
        float lam = s->slam[ci];
        float dl = (-cv - alpha * lam) / (ws + alpha);
        s->slam[ci] = lam + dl;
        float a0 = w0 * dl, a1 = -w1 * dl;
        s->p[c->v0] = vadd(p0, vmul(dir, a0));
        s->p[c->v1] = vadd(p1, vmul(dir, a1));
    }
}
/* shaders/bending.wgsl:59-126 */
static void k_bending(OSim *s, int cidx, float dt_sub) {
    uint32_t off = s->bc_off[cidx], cnt = s->bc_cnt[cidx];
#pragma omp parallel for schedule(static) if (cnt > 4096)
    for (uint32_t q = 0; q < cnt; q++) {
        uint32_t ci = off + q;
        OBend *c = &s->bend[ci];
        if (c->comp >= 1e9f) continue;
        float w2 = s->w[c->v2], w3 = s->w[c->v3];
        float ws = w2 + w3;
        if (ws <= EPS) continue;
        v3 p2 = s->p[c->v2], p3 = s->p[c->v3];
        v3 delta = vsub(p2, p3);
        float dist = vlen(delta);
        if (dist <= EPS) continue;
        if (c->pad0 > 0.5f && c->pad0 < 1.5f) {
            if (dist >= c->rest) continue;
            float gap = vlen(vsub(s->p[c->v0], s->p[c->v1]));
            if (gap > c->pad1) continue;
        }
        v3 dir = vdiv(delta, dist);
        float dt = fmaxf(dt_sub, 1e-8f);
        float alpha = c->comp / (dt * dt);
        float tau = s->bd * 1e-5f;
        float gamma = fminf(tau / dt, 1e4f);
        v3 rel = vsub(vsub(p2, s->x[c->v2]), vsub(p3, s->x[c->v3]));
        float vp = vdot(dir, rel);
        float cv = dist - c->rest;
        float lam = s->blam[ci];
        float dl = (-cv - alpha * lam - gamma * vp) / ((1.0f + gamma) * ws + alpha);
        s->blam[ci] = lam + dl;
        float a2 = w2 * dl, a3 = -w3 * dl;
        s->p[c->v2] = vadd(s->p[c->v2], vmul(dir, a2));
        s->p[c->v3] = vadd(s->p[c->v3], vmul(dir, a3));
    }
}
/* apply_contact_response, shaders/collision.wgsl:83-108 */
static void contact(v3 target, v3 nrm, float fric, float rest, float dt, v3 p_init, v3 *xn, v3 *p) {
    v3 total = vsub(target, *xn);
    v3 tang = vsub(total, vmul(nrm, vdot(total, nrm)));
    *p = vsub(target, vmul(tang, clampf(fric, 0.0f, 1.0f)));
    float edt = fmaxf(dt, 1e-6f);
    float vin = vdot(vdiv(vsub(p_init, *xn), edt), nrm);
    float des = 0.0f;
    if (vin < 0.0f) des = -clampf(rest, 0.0f, 1.0f) * vin;
    float dxn = vdot(vsub(target, *xn), nrm) - des * edt;
    *xn = vadd(*xn, vmul(nrm, dxn));
}
/* closest_point_on_triangle_ext, shaders/collision.wgsl:273-319 (and the
 * barycentric variant, shaders/self_collision.wgsl:122-166) */
static v3 closest_tri(v3 p, v3 a, v3 b, v3 c, int *is_face, v3 *bary) {
    v3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    *is_face = 0;
    if (d1 <= 0.0f && d2 <= 0.0f) { *bary = V3(1, 0, 0); return a; }
    v3 bp = vsub(p, b);
    float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) { *bary = V3(0, 1, 0); return b; }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float v = d1 / (d1 - d3);
        *bary = V3(1.0f - v, v, 0.0f);
        return vadd(a, vmul(ab, v));
    }
    v3 cp = vsub(p, c);
    float d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) { *bary = V3(0, 0, 1); return c; }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float w = d2 / (d2 - d6);
        *bary = V3(1.0f - w, 0.0f, w);
        return vadd(a, vmul(ac, w));
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        *bary = V3(0.0f, 1.0f - w, w);
        return vadd(b, vmul(vsub(c, b), w));
    }
    float denom = 1.0f / (va + vb + vc);
    float v = vb * denom, w = vc * denom;
    *is_face = 1;
    *bary = V3(1.0f - v - w, v, w);
    return vadd(vadd(a, vmul(ab, v)), vmul(ac, w));
}
/* intersect_segment_triangle, shaders/collision.wgsl:322-361 */
static int seg_tri(v3 po, v3 pn, v3 a, v3 b, v3 c, float *t_out, float *u_out, float *v_out) {
    v3 d = vsub(pn, po);
    float ld = vdot(d, d);
    if (ld < 1e-12f) return 0;
    v3 e1 = vsub(b, a), e2 = vsub(c, a);
    v3 pv = vcross(d, e2);
    float det = vdot(e1, pv);
    float tn = vdot(e1, e1) * vdot(e2, e2);
    if (det * det <= tn * ld * 1e-10f || tn <= 1e-20f) return 0;
    float inv = 1.0f / det;
    v3 tv = vsub(po, a);
    float u = vdot(tv, pv) * inv;
    if (u < -0.05f || u > 1.05f) return 0;
    v3 qv = vcross(tv, e1);
    float v = vdot(d, qv) * inv;
    if (v < -0.05f || (u + v) > 1.05f) return 0;
    float t = vdot(e2, qv) * inv;
    if (t >= 0.0f && t <= 1.0f) { *t_out = t; *u_out = u; *v_out = v; return 1; }
    return 0;
}
/* segment_sphere_dist_sq, shaders/collision.wgsl:364-375 */
static float seg_sphere_d2(v3 a, v3 b, v3 c) {
    v3 ab = vsub(b, a);
    float s2 = vdot(ab, ab);
    if (s2 <= 1e-12f) { v3 d = vsub(a, c); return vdot(d, d); }
    float t = clampf(vdot(vsub(c, a), ab) / s2, 0.0f, 1.0f);
    v3 cl = vadd(a, vmul(ab, t));
    v3 d = vsub(cl, c);
    return vdot(d, d);
}
/* one triangle of the mesh collider loop, shaders/collision.wgsl:461-541 */
static void mesh_tri(const OTri *tri, float thickness, v3 xpos, v3 *p, v3 *xn, float dt, v3 pinit,
                     int recovery_on, int *front, float *best_depth, v3 *best_pos, v3 *best_n,
                     float *best_f, float *best_r, int *has_rec) {
    float td = thickness + tri->thick;
    v3 cr = vcross(vsub(tri->p1, tri->p0), vsub(tri->p2, tri->p0));
    float cl = vlen(cr);
    if (cl < EPS) return;
    v3 fn = vdiv(cr, cl);
    int single = (tri->flags & 1u) != 0;
    float th, tu, tv;
    if (seg_tri(xpos, *p, tri->p0, tri->p1, tri->p2, &th, &tu, &tv)) {
        v3 hit = vadd(xpos, vmul(vsub(*p, xpos), th));
        v3 nn = fn;
        v3 mv = vsub(*p, xpos);
        if (vdot(mv, fn) > 0.0f && !single) nn = vneg(fn);
        v3 tgt = vadd(hit, vmul(nn, td));
        contact(tgt, nn, tri->fric, tri->rest, dt, pinit, xn, p);
        *front = 1;
    }
    int isf; v3 bary;
    v3 q = closest_tri(*p, tri->p0, tri->p1, tri->p2, &isf, &bary);
    v3 delta = vsub(*p, q);
    float dist = vlen(delta);
    float sd = vdot(delta, fn);
    if (single) {
        if (sd >= 0.0f) {
            if (dist < td) {
                v3 nn = fn;
                if (dist > EPS) nn = vdiv(delta, dist);
                v3 tgt = vadd(*p, vmul(nn, td - dist));
                contact(tgt, nn, tri->fric, tri->rest, dt, pinit, xn, p);
                *front = 1;
            }
        } else {
            int rdis = (tri->flags & 2u) != 0;
            if (recovery_on && !rdis) {
                float maxd = td * 3.0f;
                if (isf && dist < maxd && dist <= fabsf(sd) * 1.1f + EPS) {
                    if (dist < *best_depth) {
                        *best_depth = dist; *best_n = fn;
                        *best_pos = vadd(*p, vmul(fn, td - sd));
                        *best_f = tri->fric; *best_r = tri->rest; *has_rec = 1;
                    }
                }
            }
        }
    } else {
        if (dist < td && sd >= -td) {
            v3 nn = fn;
            if (dist > EPS) nn = vdiv(delta, dist);
            v3 tgt = vadd(*p, vmul(nn, td - dist));
            contact(tgt, nn, tri->fric, tri->rest, dt, pinit, xn, p);
            *front = 1;
        }
    }
}
/* shaders/collision.wgsl:378-652 (cluster culling OFF, the default) */
/* ------------------------------------------------------------------ */
/* Bone SDF: skinning.wgsl:16-43, prep_bone_triangles.wgsl:30-67,       */
/* bake_sdf.wgsl:33-196, collision.wgsl:116-265.  Matrices column-major  */
/* (row j, column k at [k*4 + j]) as GpuBoneTransform.                   */
/* ------------------------------------------------------------------ */
static inline v3 xf_point(const float *m, v3 p) {
    return V3(((m[0] * p.x + m[4] * p.y) + m[8] * p.z) + m[12], ((m[1] * p.x + m[5] * p.y) + m[9] * p.z) + m[13],
              ((m[2] * p.x + m[6] * p.y) + m[10] * p.z) + m[14]);
}
static inline v3 xf_dir(const float *m, v3 p) {
    return V3((m[0] * p.x + m[4] * p.y) + m[8] * p.z, (m[1] * p.x + m[5] * p.y) + m[9] * p.z,
              (m[2] * p.x + m[6] * p.y) + m[10] * p.z);
}
/* IEEE binary16, round to nearest even (pack2x16float) */
static uint16_t f2h(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7FFFFFFFu;
    if (ax >= 0x7F800000u) return (uint16_t)(sign | 0x7C00u | (ax > 0x7F800000u ? 0x200u : 0u));
    if (ax >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u); /* rounds to >= 65520: inf */
    if (ax < 0x38800000u) { /* subnormal half or zero */
        if (ax < 0x33000000u) return (uint16_t)sign; /* < 2^-25: rounds to 0 */
        uint32_t e = ax >> 23, m = (ax & 0x7FFFFFu) | 0x800000u;
        uint32_t shift = 126u - e; /* value = m 2^(e-150), half unit 2^-24: q = m 2^(e-126) */
        uint32_t q = m >> shift, rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1u);
        if (rem > half || (rem == half && (q & 1u))) q++;
        return (uint16_t)(sign | q);
    }
    uint32_t e = (ax >> 23) - 112u, m = ax & 0x7FFFFFu;
    uint32_t q = (e << 10) | (m >> 13), rem = m & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q++;
    return (uint16_t)(sign | q);
}
static float h2f(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1Fu, m = h & 0x3FFu, x;
    if (e == 0) {
        if (m == 0) x = sign;
        else { float f = ldexpf((float)m, -24); memcpy(&x, &f, 4); x |= sign; }
    } else if (e == 31) x = sign | 0x7F800000u | (m << 13);
    else x = sign | ((e + 112u) << 23) | (m << 13);
    float f;
    memcpy(&f, &x, 4);
    return f;
}
void ocl_half_roundtrip(const float *in, int n, uint16_t *bits, float *out) {
    for (int i = 0; i < n; i++) { bits[i] = f2h(in[i]); out[i] = h2f(bits[i]); }
}

/* Host product of mod.rs:2339-2345: S = transpose(transpose(W) * B), W column-major, B row-major */
void ocl_bone_skin_mats(int nb, const float *world, const float *bind_inv, float *out) {
    for (int b = 0; b < nb; b++) {
        float wr[4][4], bb[4][4], sr[4][4];
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) { wr[i][j] = world[32 * b + j * 4 + i]; bb[i][j] = bind_inv[16 * b + i * 4 + j]; }
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++)
                sr[i][j] = ((wr[i][0] * bb[0][j] + wr[i][1] * bb[1][j]) + wr[i][2] * bb[2][j]) + wr[i][3] * bb[3][j];
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) out[16 * b + i * 4 + j] = sr[j][i];
    }
}
void ocl_bone_skin(int nv, const float *rest4, const uint32_t *bidx, const float *bw, const float *skin_mats,
                   float *out4) {
    for (int i = 0; i < nv; i++) {
        v3 pos = V3(rest4[4 * i], rest4[4 * i + 1], rest4[4 * i + 2]);
        v3 p = V3(0, 0, 0);
        float ws = 0.0f;
        for (int k = 0; k < 4; k++) {
            float w = bw[4 * i + k];
            if (w > 0.0f) {
                p = vadd(p, vmul(xf_point(skin_mats + 16 * (size_t)bidx[4 * i + k], pos), w));
                ws += w;
            }
        }
        if (ws <= 1e-6f) p = pos;
        out4[4 * i] = p.x; out4[4 * i + 1] = p.y; out4[4 * i + 2] = p.z; out4[4 * i + 3] = 1.0f;
    }
}
void ocl_bone_prep(int nt, const float *skinned4, const float *inv_mats, const uint32_t *src, const float *srcw,
                   float *out16) {
    for (int t = 0; t < nt; t++) {
        const uint32_t *q = src + 4 * t;
        const float *inv = inv_mats + 16 * (size_t)q[3];
        v3 p0 = xf_point(inv, V3(skinned4[4 * q[0]], skinned4[4 * q[0] + 1], skinned4[4 * q[0] + 2]));
        v3 p1 = xf_point(inv, V3(skinned4[4 * q[1]], skinned4[4 * q[1] + 1], skinned4[4 * q[1] + 2]));
        v3 p2 = xf_point(inv, V3(skinned4[4 * q[2]], skinned4[4 * q[2] + 1], skinned4[4 * q[2] + 2]));
        v3 cr = vcross(vsub(p1, p0), vsub(p2, p0));
        float l2 = vdot(cr, cr);
        v3 nrm = V3(0.0f, 1.0f, 0.0f);
        if (l2 > 1e-12f) nrm = vmul(cr, 1.0f / sqrtf(l2));
        float *o = out16 + 16 * t;
        o[0] = p0.x; o[1] = p0.y; o[2] = p0.z; o[3] = srcw[4 * t];
        o[4] = p1.x; o[5] = p1.y; o[6] = p1.z; o[7] = srcw[4 * t + 1];
        o[8] = p2.x; o[9] = p2.y; o[10] = p2.z; o[11] = srcw[4 * t + 2];
        o[12] = nrm.x; o[13] = nrm.y; o[14] = nrm.z; o[15] = srcw[4 * t + 3];
    }
}
/* bake_mesh_sdf_gpu without boundary capping (closed meshes):
 * mesh_sdf_domain / mesh_sdf_bone_info / collect_mesh_bake_triangles
 * (sdf_baker.rs:939-1060) and bake_mesh_sdf.wgsl, every triangle of every
 * voxel in order.  dims and info are written; texels (w x h x d) when given. */
/* mesh_sdf_domain / mesh_sdf_bone_info, sdf_baker.rs:939-1016 */
static void mesh_domain(const float *verts, int nv, float voxel, float margin, float friction, float thickness,
                        float restitution, float *lo, float *hi, float *size, uint32_t *dims, float *info) {
    for (int k = 0; k < 3; k++) { lo[k] = INFINITY; hi[k] = -INFINITY; }
    for (int v = 0; v < nv; v++)
        for (int k = 0; k < 3; k++) { lo[k] = fminf(lo[k], verts[3 * v + k]); hi[k] = fmaxf(hi[k], verts[3 * v + k]); }
    float vs = fmaxf(voxel, 0.001f);
    for (int k = 0; k < 3; k++) {
        size[k] = fmaxf(hi[k] - lo[k], 0.05f);
        float pad = fmaxf(size[k] * margin, 0.04f) + fmaxf(thickness, 0.0f) + 0.02f;
        lo[k] -= pad; hi[k] += pad;
        size[k] = hi[k] - lo[k];
        float raw = ceilf(size[k] / vs);
        double r = (raw == raw && raw > 0.0f) ? (double)raw : 0.0;
        dims[k] = (uint32_t)(r < 8.0 ? 8.0 : (r > 2048.0 ? 2048.0 : r));
    }
    if (!info) return;
    for (int k = 0; k < 20; k++) info[k] = 0.0f;
    for (int k = 0; k < 3; k++) {
        info[k] = lo[k]; info[4 + k] = hi[k]; info[8 + k] = 1.0f / size[k]; info[12 + k] = -lo[k] / size[k];
    }
    info[7] = (float)dims[0]; info[16] = friction; info[17] = thickness; info[18] = restitution;
}
/* collect_mesh_bake_triangles, sdf_baker.rs:1018-1060: 12 floats per valid
 * triangle (corners, unit normal; zero cross product: (0, 1, 0)); at least
 * one (degenerate) entry.  *m = count. */
static float *mesh_tris12(const float *verts, int nv, const int32_t *tris, int nt, int *m_out) {
    float *T = (float *)malloc(sizeof(float) * 12 * ((size_t)nt + 1));
    int m = 0;
    for (int t = 0; t < nt; t++) {
        int i0 = tris[3 * t], i1 = tris[3 * t + 1], i2 = tris[3 * t + 2];
        if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= nv || i1 >= nv || i2 >= nv) continue;
        const float *p0 = verts + 3 * i0, *p1 = verts + 3 * i1, *p2 = verts + 3 * i2;
        v3 a = V3(p0[0], p0[1], p0[2]), b = V3(p1[0], p1[1], p1[2]), c = V3(p2[0], p2[1], p2[2]);
        v3 cr = vcross(vsub(b, a), vsub(c, a));
        float l2 = cr.x * cr.x + cr.y * cr.y + cr.z * cr.z;
        v3 n = V3(0.0f, 1.0f, 0.0f);
        if (l2 > 1e-12f) { float il = 1.0f / sqrtf(l2); n = V3(cr.x * il, cr.y * il, cr.z * il); }
        float *q = T + 12 * m++;
        q[0] = a.x; q[1] = a.y; q[2] = a.z; q[3] = b.x; q[4] = b.y; q[5] = b.z;
        q[6] = c.x; q[7] = c.y; q[8] = c.z; q[9] = n.x; q[10] = n.y; q[11] = n.z;
    }
    if (m == 0) { memset(T, 0, 12 * sizeof(float)); T[10] = 1.0f; m = 1; }
    *m_out = m;
    return T;
}
/* closest_point_on_triangle + sign by the normal, bake_mesh_sdf.wgsl and
 * bake_mesh_sdf_hier_common.wgsl:30-78: squared distance, *sd = signed distance */
static float tri_sdist(v3 p, const float *q, float *sd) {
    v3 a = V3(q[0], q[1], q[2]), b = V3(q[3], q[4], q[5]), c = V3(q[6], q[7], q[8]);
    v3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a), cp;
    float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    v3 bp = vsub(p, b);
    float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    v3 cpv = vsub(p, c);
    float d5 = vdot(ab, cpv), d6 = vdot(ac, cpv);
    float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
    if (d1 <= 0.0f && d2 <= 0.0f) cp = a;
    else if (d3 >= 0.0f && d4 <= d3) cp = b;
    else if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) cp = vadd(a, vmul(ab, d1 / (d1 - d3)));
    else if (d6 >= 0.0f && d5 <= d6) cp = c;
    else if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) cp = vadd(a, vmul(ac, d2 / (d2 - d6)));
    else if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f)
        cp = vadd(b, vmul(vsub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
    else {
        float den = 1.0f / (va + vb + vc);
        cp = vadd(vadd(a, vmul(ab, vb * den)), vmul(ac, vc * den));
    }
    v3 diff = vsub(p, cp);
    float dsq = vdot(diff, diff);
    *sd = sqrtf(dsq) * (vdot(diff, V3(q[9], q[10], q[11])) >= 0.0f ? 1.0f : -1.0f);
    return dsq;
}
static inline v3 voxel_centre(const float *lo, const float *hi, uint32_t x, uint32_t y, uint32_t z, uint32_t W,
                              uint32_t H, uint32_t D) {
    float iw = 1.0f / (float)W, ih = 1.0f / (float)H, id = 1.0f / (float)D;
    return V3(lo[0] + ((float)x + 0.5f) * iw * (hi[0] - lo[0]), lo[1] + ((float)y + 0.5f) * ih * (hi[1] - lo[1]),
              lo[2] + ((float)z + 0.5f) * id * (hi[2] - lo[2]));
}
static inline uint32_t pack_h2(float a, float b) { return (uint32_t)f2h(a) | ((uint32_t)f2h(b) << 16); }

/* Single-mesh SDF of an already capped mesh (bake_mesh_sdf_gpu_ext without
 * capping): mesh_sdf_domain / mesh_sdf_bone_info / collect_mesh_bake_triangles
 * (sdf_baker.rs:939-1060) and bake_mesh_sdf.wgsl, every triangle of every
 * voxel in order.  dims and info are written; texels (w x h x d) when given. */
void ocl_bake_mesh_sdf(const float *verts, int nv, const int32_t *tris, int nt, float voxel, float margin,
                       float friction, float thickness, float restitution, uint32_t *dims, float *info,
                       uint32_t *texels) {
    float lo[3], hi[3], size[3];
    mesh_domain(verts, nv, voxel, margin, friction, thickness, restitution, lo, hi, size, dims, info);
    if (!texels) return;
    int m;
    float *T = mesh_tris12(verts, nv, tris, nt, &m);
    uint32_t W = dims[0], H = dims[1], D = dims[2];
#pragma omp parallel for schedule(dynamic, 4)
    for (int z = 0; z < (int)D; z++)
        for (uint32_t y = 0; y < H; y++)
            for (uint32_t x = 0; x < W; x++) {
                v3 p = voxel_centre(lo, hi, x, y, (uint32_t)z, W, H, D);
                float md = 1e10f, best = 10.0f;
                for (int t = 0; t < m; t++) {
                    float sd, dsq = tri_sdist(p, T + 12 * t, &sd);
                    if (dsq < md) { md = dsq; best = sd; }
                }
                texels[((size_t)z * H + y) * W + x] = pack_h2(best, 1.0f);
            }
    free(T);
}

/* Coarse pass of the hierarchical bake (bake_mesh_sdf_coarse_ext without
 * capping, sdf_baker.rs:1350-1600; bake_mesh_sdf_hier_coarse_main.wgsl):
 * domain at max(voxel x 4, 0.001); per voxel the 8 nearest triangles by an
 * in-order insertion with strict <; dist = fp16 (signed distance of the
 * first, 1), near8[voxel * 8 + k].  dims and *coarse_voxel always written. */
void ocl_bake_mesh_sdf_coarse(const float *verts, int nv, const int32_t *tris, int nt, float voxel, float margin,
                              float thickness, uint32_t *dims, float *coarse_voxel, uint32_t *dist, uint32_t *near8) {
    float lo[3], hi[3], size[3];
    float cv = fmaxf(voxel * 4.0f, 0.001f);
    *coarse_voxel = cv;
    mesh_domain(verts, nv, cv, margin, 0.0f, thickness, 0.0f, lo, hi, size, dims, NULL);
    if (!dist) return;
    int m;
    float *T = mesh_tris12(verts, nv, tris, nt, &m);
    uint32_t W = dims[0], H = dims[1], D = dims[2];
#pragma omp parallel for schedule(dynamic, 1)
    for (int z = 0; z < (int)D; z++)
        for (uint32_t y = 0; y < H; y++)
            for (uint32_t x = 0; x < W; x++) {
                v3 p = voxel_centre(lo, hi, x, y, (uint32_t)z, W, H, D);
                float bsq[8], bsg[8];
                uint32_t bid[8];
                for (int k = 0; k < 8; k++) { bsq[k] = 1e10f; bsg[k] = 10.0f; bid[k] = 0u; }
                for (int t = 0; t < m; t++) {
                    float sd, dsq = tri_sdist(p, T + 12 * t, &sd);
                    if (dsq < bsq[7]) {
                        float isq = dsq, isg = sd;
                        uint32_t iid = (uint32_t)t;
                        for (int k = 0; k < 8; k++) {
                            if (isq < bsq[k]) {
                                float tq = bsq[k], ts = bsg[k];
                                uint32_t ti = bid[k];
                                bsq[k] = isq; bsg[k] = isg; bid[k] = iid;
                                isq = tq; isg = ts; iid = ti;
                            }
                        }
                    }
                }
                size_t flat = ((size_t)z * H + y) * W + x;
                dist[flat] = pack_h2(bsg[0], 1.0f);
                for (int k = 0; k < 8; k++) near8[flat * 8 + k] = bid[k];
            }
    free(T);
}

/* Hierarchical bake of an already capped mesh (bake_mesh_sdf_hierarchical_ext
 * without capping, sdf_baker.rs:1625-1900; bake_mesh_sdf_hier_fine_main.wgsl).
 * Returns 0, or 1 when the band is wider than two coarse cells (the
 * reference's error).  dims and info written; texels when given. */
int ocl_bake_mesh_sdf_hier(const float *verts, int nv, const int32_t *tris, int nt, float voxel, float margin,
                           float friction, float thickness, float restitution, uint32_t *dims, float *info,
                           uint32_t *texels) {
    float lo[3], hi[3], size[3];
    mesh_domain(verts, nv, voxel, margin, friction, thickness, restitution, lo, hi, size, dims, info);
    uint32_t cd[3];
    float cv;
    ocl_bake_mesh_sdf_coarse(verts, nv, tris, nt, voxel, margin, thickness, cd, &cv, NULL, NULL);
    float h_fine = fmaxf(fmaxf(size[0] / (float)dims[0], size[1] / (float)dims[1]), size[2] / (float)dims[2]);
    float band = 4.0f * h_fine;
    float hcm = fminf(fminf(size[0] / (float)cd[0], size[1] / (float)cd[1]), size[2] / (float)cd[2]);
    if (band > 2.0f * hcm) return 1;
    if (!texels) return 0;
    size_t ncv = (size_t)cd[0] * cd[1] * cd[2];
    uint32_t *cdist = (uint32_t *)malloc(4 * ncv), *cnear = (uint32_t *)malloc(32 * ncv);
    ocl_bake_mesh_sdf_coarse(verts, nv, tris, nt, voxel, margin, thickness, cd, &cv, cdist, cnear);
    int m;
    float *T = mesh_tris12(verts, nv, tris, nt, &m);
    uint32_t W = dims[0], H = dims[1], D = dims[2];
    v3 vlo = V3(lo[0], lo[1], lo[2]);
    v3 sz = vsub(V3(hi[0], hi[1], hi[2]), vlo);
    v3 cdf = V3((float)cd[0], (float)cd[1], (float)cd[2]);
    v3 spacing = V3(sz.x / cdf.x, sz.y / cdf.y, sz.z / cdf.z);
    float halfdiag = 0.5f * vlen(spacing);
    int32_t hx = (int32_t)cd[0] - 1, hy = (int32_t)cd[1] - 1, hz = (int32_t)cd[2] - 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int z = 0; z < (int)D; z++)
        for (uint32_t y = 0; y < H; y++)
            for (uint32_t x = 0; x < W; x++) {
                float iw = 1.0f / (float)W, ih = 1.0f / (float)H, id = 1.0f / (float)D;
                v3 p = V3(vlo.x + ((float)x + 0.5f) * iw * sz.x, vlo.y + ((float)y + 0.5f) * ih * sz.y,
                          vlo.z + ((float)z + 0.5f) * id * sz.z);
                v3 rel = vsub(p, vlo);
                int32_t px = f2i(floorf(rel.x / spacing.x)), py = f2i(floorf(rel.y / spacing.y)),
                        pz = f2i(floorf(rel.z / spacing.z));
                px = px < 0 ? 0 : (px > hx ? hx : px);
                py = py < 0 ? 0 : (py > hy ? hy : py);
                pz = pz < 0 ? 0 : (pz > hz ? hz : pz);
                size_t flat = ((size_t)z * H + y) * W + x;
                uint32_t pidx = ((uint32_t)pz * cd[1] + (uint32_t)py) * cd[0] + (uint32_t)px;
                uint32_t dcp = cdist[pidx];
                float dc = h2f((uint16_t)(dcp & 0xFFFFu));
                if (fabsf(dc) - halfdiag >= band) { texels[flat] = dcp; continue; }
                uint32_t bi = 0xFFFFFFFFu;
                float bsq = 1e10f, bsg = 10.0f, ssq = 1e10f, ssg = 10.0f;
                for (int dz = -2; dz <= 2; dz++)
                    for (int dy = -2; dy <= 2; dy++)
                        for (int dx = -2; dx <= 2; dx++) {
                            int32_t cx = px + dx, cy = py + dy, cz = pz + dz;
                            cx = cx < 0 ? 0 : (cx > hx ? hx : cx);
                            cy = cy < 0 ? 0 : (cy > hy ? hy : cy);
                            cz = cz < 0 ? 0 : (cz > hz ? hz : cz);
                            size_t base = (((size_t)cz * cd[1] + (size_t)cy) * cd[0] + (size_t)cx) * 8u;
                            for (int k = 0; k < 8; k++) {
                                uint32_t ti = cnear[base + k];
                                if (ti >= (uint32_t)m || ti == bi) continue;
                                const float *q = T + 12 * (size_t)ti;
                                v3 a = V3(q[0], q[1], q[2]), b = V3(q[3], q[4], q[5]), c = V3(q[6], q[7], q[8]);
                                v3 tmin = vmin(a, vmin(b, c)), tmax = vmax(a, vmax(b, c));
                                v3 dv = vadd(vmax(vsub(tmin, p), V3(0, 0, 0)), vmax(vsub(p, tmax), V3(0, 0, 0)));
                                if (vdot(dv, dv) >= ssq) continue;
                                float sd, dsq = tri_sdist(p, q, &sd);
                                if (dsq < bsq) { ssq = bsq; ssg = bsg; bsq = dsq; bsg = sd; bi = ti; }
                                else if (dsq < ssq) { ssq = dsq; ssg = sd; }
                            }
                        }
                int amb = (sqrtf(ssq) - sqrtf(bsq) <= 0.0002f);
                if (amb) {
                    float sb = bsg >= 0.0f ? 1.0f : -1.0f, ss = ssg >= 0.0f ? 1.0f : -1.0f;
                    amb = sb != ss;
                }
                if (amb) {
                    bsq = 1e10f; bsg = 10.0f;
                    for (int t = 0; t < m; t++) {
                        float sd, dsq = tri_sdist(p, T + 12 * t, &sd);
                        if (dsq < bsq) { bsq = dsq; bsg = sd; }
                    }
                }
                texels[flat] = pack_h2(bsg, 1.0f);
            }
    free(T); free(cdist); free(cnear);
    return 0;
}

/* params: 16 words per bone (GpuBakeParams); every triangle of the bone in order */
void ocl_bone_bake(int np, const uint32_t *params, const float *tris16, uint32_t *atlas) {
    for (int bi = 0; bi < np; bi++) {
        const uint32_t *P = params + 16 * bi;
        float lmin[3], lmax[3];
        memcpy(lmin, P, 12);
        memcpy(lmax, P + 4, 12);
        uint32_t tri_start = P[3], tri_count = P[7], col = P[8], row = P[9], layer = P[10], res = P[11];
        uint32_t tw = P[12], th = P[13], pitch_w = P[15] > 0 ? P[15] : tw;
        float fr = (float)res;
#pragma omp parallel for collapse(2) schedule(static)
        for (uint32_t vz = 0; vz < res; vz++)
            for (uint32_t vy = 0; vy < res; vy++)
                for (uint32_t vx = 0; vx < res; vx++) {
                    v3 uvw = V3(((float)vx + 0.5f) / fr, ((float)vy + 0.5f) / fr, ((float)vz + 0.5f) / fr);
                    v3 p = V3(lmin[0] + uvw.x * (lmax[0] - lmin[0]), lmin[1] + uvw.y * (lmax[1] - lmin[1]),
                              lmin[2] + uvw.z * (lmax[2] - lmin[2]));
                    float min_d2 = 1e10f, bap = -1.0f, bsd = 10.0f, bal = 0.0f;
                    for (uint32_t i = 0; i < tri_count; i++) {
                        const float *T = tris16 + 16 * (size_t)(tri_start + i);
                        v3 a = V3(T[0], T[1], T[2]), b = V3(T[4], T[5], T[6]), c = V3(T[8], T[9], T[10]);
                        v3 nrm = V3(T[12], T[13], T[14]);
                        v3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
                        float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
                        v3 cp = a, bary = V3(1, 0, 0);
                        if (d1 <= 0.0f && d2 <= 0.0f) {
                        } else {
                            v3 bp = vsub(p, b);
                            float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
                            if (d3 >= 0.0f && d4 <= d3) { cp = b; bary = V3(0, 1, 0); }
                            else {
                                float vc = d1 * d4 - d3 * d2;
                                if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
                                    float v = d1 / (d1 - d3);
                                    cp = vadd(a, vmul(ab, v)); bary = V3(1.0f - v, v, 0);
                                } else {
                                    v3 cpv = vsub(p, c);
                                    float d5 = vdot(ab, cpv), d6 = vdot(ac, cpv);
                                    if (d6 >= 0.0f && d5 <= d6) { cp = c; bary = V3(0, 0, 1); }
                                    else {
                                        float vb = d5 * d2 - d1 * d6;
                                        if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
                                            float w = d2 / (d2 - d6);
                                            cp = vadd(a, vmul(ac, w)); bary = V3(1.0f - w, 0, w);
                                        } else {
                                            float va = d3 * d6 - d5 * d4;
                                            if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
                                                float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
                                                cp = vadd(b, vmul(vsub(c, b), w)); bary = V3(0, 1.0f - w, w);
                                            } else {
                                                float denom = 1.0f / ((va + vb) + vc);
                                                float v = vb * denom, w = vc * denom;
                                                float u = (1.0f - v) - w;
                                                cp = vadd(vadd(a, vmul(ab, v)), vmul(ac, w));
                                                bary = V3(u, v, w);
                                            }
                                        }
                                    }
                                }
                            }
                        }
                        v3 diff = vsub(p, cp);
                        float d_sq = vdot(diff, diff);
                        float proj = vdot(diff, nrm), aproj = fabsf(proj);
                        float eps_sq = 1e-7f * fmaxf(1.0f, min_d2);
                        int closer = d_sq + eps_sq < min_d2;
                        int tie = fabsf(d_sq - min_d2) <= eps_sq && aproj > bap;
                        if (closer || tie) {
                            if (d_sq < min_d2) min_d2 = d_sq;
                            bap = aproj;
                            float d = sqrtf(d_sq);
                            float sign = proj >= 0.0f ? 1.0f : -1.0f;
                            uint32_t bmask = (uint32_t)(T[15] + 0.5f);
                            if (bmask != 0u && sign < 0.0f) {
                                float op = -1.0f;
                                if ((bmask & 1u) && bary.z <= 1e-5f) {
                                    v3 e = vcross(vsub(b, a), nrm);
                                    op = fmaxf(op, vdot(diff, vdiv(e, vlen(e))));
                                }
                                if ((bmask & 2u) && bary.x <= 1e-5f) {
                                    v3 e = vcross(vsub(c, b), nrm);
                                    op = fmaxf(op, vdot(diff, vdiv(e, vlen(e))));
                                }
                                if ((bmask & 4u) && bary.y <= 1e-5f) {
                                    v3 e = vcross(vsub(a, c), nrm);
                                    op = fmaxf(op, vdot(diff, vdiv(e, vlen(e))));
                                }
                                if (op > 0.0f && op >= aproj * 0.25f) sign = 1.0f;
                            }
                            bsd = d * sign;
                            bal = (bary.x * T[3] + bary.y * T[7]) + bary.z * T[11];
                        }
                    }
                    uint32_t gx = col * res + vx, gy = row * res + vy, gz = layer * res + vz;
                    atlas[((size_t)gz * th + gy) * pitch_w + gx] = (uint32_t)f2h(bsd) | ((uint32_t)f2h(bal) << 16);
                }
    }
}
void ocl_set_bone_sdf(OSim *s, uint32_t w, uint32_t h, uint32_t d, const uint32_t *atlas, int nbones,
                      const float *infos20, const float *xforms32) {
    free(s->atlas); free(s->binfo); free(s->bxf);
    s->atlas = NULL; s->binfo = NULL; s->bxf = NULL; s->nbones = 0;
    if (nbones <= 0) return;
    size_t nvox = (size_t)w * h * d;
    s->atlas = malloc(nvox * 4); memcpy(s->atlas, atlas, nvox * 4);
    s->binfo = malloc((size_t)nbones * 20 * 4); memcpy(s->binfo, infos20, (size_t)nbones * 20 * 4);
    s->bxf = malloc((size_t)nbones * 32 * 4); memcpy(s->bxf, xforms32, (size_t)nbones * 32 * 4);
    s->aw = w; s->ah = h; s->ad = d; s->nbones = nbones;
}
static void atlas_at(const OSim *s, int x, int y, int z, float *dv, float *av) {
    uint32_t u = s->atlas[((size_t)z * s->ah + y) * s->aw + x];
    *dv = h2f((uint16_t)(u & 0xFFFFu));
    *av = h2f((uint16_t)(u >> 16));
}
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
/* trilinear, clamp to edge, fp32 weights */
static void sample_atlas(const OSim *s, v3 uvw, float *dist, float *alpha) {
    float fx = uvw.x * (float)s->aw - 0.5f, fy = uvw.y * (float)s->ah - 0.5f, fz = uvw.z * (float)s->ad - 0.5f;
    float flx = floorf(fx), fly = floorf(fy), flz = floorf(fz);
    float tx = fx - flx, ty = fy - fly, tz = fz - flz;
    int ix = (int)flx, iy = (int)fly, iz = (int)flz;
    int x0 = clampi(ix, 0, (int)s->aw - 1), x1 = clampi(ix + 1, 0, (int)s->aw - 1);
    int y0 = clampi(iy, 0, (int)s->ah - 1), y1 = clampi(iy + 1, 0, (int)s->ah - 1);
    int z0 = clampi(iz, 0, (int)s->ad - 1), z1 = clampi(iz + 1, 0, (int)s->ad - 1);
    float rz[2][2];
    for (int zi = 0; zi < 2; zi++) {
        int z = zi ? z1 : z0;
        float ry[2][2];
        for (int yi = 0; yi < 2; yi++) {
            int y = yi ? y1 : y0;
            float pd, pa, qd, qa;
            atlas_at(s, x0, y, z, &pd, &pa);
            atlas_at(s, x1, y, z, &qd, &qa);
            ry[yi][0] = pd * (1.0f - tx) + qd * tx;
            ry[yi][1] = pa * (1.0f - tx) + qa * tx;
        }
        rz[zi][0] = ry[0][0] * (1.0f - ty) + ry[1][0] * ty;
        rz[zi][1] = ry[0][1] * (1.0f - ty) + ry[1][1] * ty;
    }
    *dist = rz[0][0] * (1.0f - tz) + rz[1][0] * tz;
    *alpha = rz[0][1] * (1.0f - tz) + rz[1][1] * tz;
}
static float sample_d(const OSim *s, v3 uvw) { float d, a; sample_atlas(s, uvw, &d, &a); return d; }
static float smoothstep_f(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return (t * t) * (3.0f - 2.0f * t);
}
static int bone_sdf_contact(const OSim *s, v3 p, float vth, v3 *target, v3 *nrm_out, float *fric, float *rest) {
    float best = 1e6f, best_target = 0.0f, bf = 0.0f, br = 0.0f;
    v3 best_n = V3(0, 0, 0);
    unsigned hits = 0;
    int has_mesh = s->ntris > 0;
    for (int b = 0; b < s->nbones; b++) {
        const float *I = s->binfo + 20 * b;
        const float *X = s->bxf + 32 * b;
        float wr = I[15];
        if (wr > 0.0f) {
            v3 dw = vsub(p, V3(I[3], I[7], I[11]));
            float rt = wr + vth;
            if (vdot(dw, dw) > rt * rt) continue;
        }
        v3 pl = xf_point(X + 16, p);
        float target_dist = vth + I[17];
        float margin = target_dist + 0.05f;
        if (pl.x < I[0] - margin || pl.x > I[4] + margin || pl.y < I[1] - margin || pl.y > I[5] + margin ||
            pl.z < I[2] - margin || pl.z > I[6] + margin)
            continue;
        v3 sc = V3(I[8], I[9], I[10]), of = V3(I[12], I[13], I[14]);
        v3 uvw = V3(pl.x * sc.x + of.x, pl.y * sc.y + of.y, pl.z * sc.z + of.z);
        v3 umin = V3(I[0] * sc.x + of.x, I[1] * sc.y + of.y, I[2] * sc.z + of.z);
        v3 umax = V3(I[4] * sc.x + of.x, I[5] * sc.y + of.y, I[6] * sc.z + of.z);
        if (uvw.x < umin.x || uvw.x > umax.x || uvw.y < umin.y || uvw.y > umax.y || uvw.z < umin.z || uvw.z > umax.z)
            continue;
        v3 es = vmul(vsub(umax, umin), s->nbones == 1 ? 0.002f : 0.015f);
        v3 lo = vadd(umin, es), hi = vsub(umax, es);
        v3 us = V3(clampf(uvw.x, lo.x, hi.x), clampf(uvw.y, lo.y, hi.y), clampf(uvw.z, lo.z, hi.z));
        float raw, alpha;
        sample_atlas(s, us, &raw, &alpha);
        float thr = fmaxf(I[19], 0.01f);
        float retract = 0.0f;
        if (has_mesh) retract = (1.0f - smoothstep_f(thr, 0.7f, alpha)) * 0.06f;
        float eff = alpha > thr ? raw + retract : 10.0f;
        if (eff < target_dist) {
            v3 eu = vmul(sc, 0.005f);
            float dxp = sample_d(s, V3(clampf(uvw.x + eu.x, lo.x, hi.x), us.y, us.z));
            float dxn = sample_d(s, V3(clampf(uvw.x - eu.x, lo.x, hi.x), us.y, us.z));
            float dyp = sample_d(s, V3(us.x, clampf(uvw.y + eu.y, lo.y, hi.y), us.z));
            float dyn = sample_d(s, V3(us.x, clampf(uvw.y - eu.y, lo.y, hi.y), us.z));
            float dzp = sample_d(s, V3(us.x, us.y, clampf(uvw.z + eu.z, lo.z, hi.z)));
            float dzn = sample_d(s, V3(us.x, us.y, clampf(uvw.z - eu.z, lo.z, hi.z)));
            float dx = dxp - dxn, dy = dyp - dyn, dz = dzp - dzn;
            if (fabsf(dx) < 1e-6f) dx = uvw.x < (lo.x + hi.x) * 0.5f ? dxp - raw : raw - dxn;
            if (fabsf(dy) < 1e-6f) dy = uvw.y < (lo.y + hi.y) * 0.5f ? dyp - raw : raw - dyn;
            if (fabsf(dz) < 1e-6f) dz = uvw.z < (lo.z + hi.z) * 0.5f ? dzp - raw : raw - dzn;
            v3 g = V3(dx, dy, dz);
            float gl = vlen(g);
            v3 nl = V3(0, 0, 1);
            if (gl > 1e-6f) nl = vdiv(g, gl);
            else {
                v3 cl = vmul(vadd(V3(I[0], I[1], I[2]), V3(I[4], I[5], I[6])), 0.5f);
                v3 dc = vsub(pl, cl);
                float lc = vlen(dc);
                if (lc > 1e-6f) nl = vdiv(dc, lc);
            }
            v3 nwr = xf_dir(X, nl);
            v3 nw = vdiv(nwr, vlen(nwr));
            if (hits == 0 || eff < best) { best = eff; best_n = nw; bf = I[16]; br = I[18]; best_target = target_dist; }
            hits++;
        }
    }
    if (hits > 0 && best < best_target) {
        *target = vadd(p, vmul(best_n, best_target - best));
        *nrm_out = best_n;
        *fric = bf;
        *rest = br;
        return 1;
    }
    return 0;
}

static void k_collision(OSim *s, float dt) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < s->n; i++) {
        if (s->w[i] <= 0.0f) continue;
        v3 p = s->p[i];
        v3 pinit = p;
        v3 xn = s->x[i];
        v3 xpos = s->x[i];
        float th = s->thick[i];
        for (int k = 0; k < s->ncols; k++) {
            OCol *c = &s->cols[k];
            if (c->type == 0) {
                float tr = c->r + th;
                v3 d = vsub(p, c->a);
                float dist = vlen(d);
                if (dist < tr) {
                    v3 nn = V3(0, 0, 1);
                    if (dist > EPS) nn = vdiv(d, dist);
                    v3 tgt = vadd(c->a, vmul(nn, tr));
                    contact(tgt, nn, c->fric, c->rest, dt, pinit, &xn, &p);
                }
            } else if (c->type == 1) {
                float tr = c->r + th;
                v3 ab = vsub(c->b, c->a);
                float l2 = vdot(ab, ab);
                float t = 0.0f;
                if (l2 > EPS) t = clampf(vdot(vsub(p, c->a), ab) / l2, 0.0f, 1.0f);
                v3 cl = vadd(c->a, vmul(ab, t));
                v3 d = vsub(p, cl);
                float dist = vlen(d);
                if (dist < tr) {
                    v3 nn = V3(0, 0, 1);
                    if (dist > EPS) nn = vdiv(d, dist);
                    v3 tgt = vadd(cl, vmul(nn, tr));
                    contact(tgt, nn, c->fric, c->rest, dt, pinit, &xn, &p);
                }
            } else if (c->type == 2) {
                v3 pn = vdiv(c->b, vlen(c->b));
                float dist = vdot(vsub(p, c->a), pn);
                if (dist < th) {
                    v3 tgt = vadd(p, vmul(pn, th - dist));
                    contact(tgt, pn, c->fric, c->rest, dt, pinit, &xn, &p);
                }
            }
        }
        int front = 0, hasrec = 0;
        float bdepth = 999999.0f, bf = 0.0f, br = 0.0f;
        v3 bpos = p, bn = V3(0, 0, 0);
        for (int t = 0; t < s->ntris; t++) {
            const float *b = s->bounds + 4 * t;
            float r = b[3] * 1.5f + th;
            if (seg_sphere_d2(xpos, p, V3(b[0], b[1], b[2])) > r * r) continue;
            mesh_tri(&s->tris[t], th, xpos, &p, &xn, dt, pinit, s->single_sided_recovery, &front, &bdepth,
                     &bpos, &bn, &bf, &br, &hasrec);
        }
        if (!front && hasrec) contact(bpos, bn, bf, br, dt, pinit, &xn, &p);
        if (s->nbones > 0) {
            v3 tgt, bnn;
            float bfr, brs;
            if (bone_sdf_contact(s, p, th, &tgt, &bnn, &bfr, &brs)) {
                v3 pb = p;
                contact(tgt, bnn, bfr, brs, dt, pb, &xn, &p);
            }
        }
        s->p[i] = p;
        s->x[i] = xn;
    }
}
/* shaders/update_vel.wgsl:33-53 */
static void k_update_vel(OSim *s, float dt_sub) {
    float dt = fmaxf(dt_sub, 1e-8f);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; i++) {
        if (s->w[i] > 0.0f) s->v[i] = vdiv(vsub(s->p[i], s->x[i]), dt);
        else s->v[i] = V3(0, 0, 0);
        s->x[i] = s->p[i];
    }
}
/* shaders/compute_normals.wgsl:25-58 */
static void k_normals(OSim *s) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; i++) {
        v3 pi = s->x[i];
        v3 sum = V3(0, 0, 0);
        for (uint32_t k = s->star_off[i]; k < s->star_off[i + 1]; k++) {
            v3 pa = s->x[s->star_idx[2 * k]], pb = s->x[s->star_idx[2 * k + 1]];
            sum = vadd(sum, vcross(vsub(pa, pi), vsub(pb, pi)));
        }
        float l = vlen(sum);
        s->nrm[i] = l > EPS ? vdiv(sum, l) : V3(0, 0, 0);
    }
}
/* hash_coords, shaders/spatial_grid_sort.wgsl:25-31 */
static inline uint32_t hash3(int32_t cx, int32_t cy, int32_t cz, uint32_t table) {
    uint32_t h = ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^ ((uint32_t)cz * 83492791u);
    return h % table;
}
static inline void cell_of(v3 p, float cell, int32_t *c) {
    c[0] = f2i(floorf(p.x / cell)); c[1] = f2i(floorf(p.y / cell)); c[2] = f2i(floorf(p.z / cell));
}
/* six-phase counting sort, spatial_hash.rs:158-247 with
 * shaders/spatial_grid_sort.wgsl:34-195 (vertex keys) and
 * shaders/spatial_grid_sort_edges.wgsl:40-200 (edge midpoint keys).
 * Within a bucket: ascending index (canonical order). */
static void build_hash(OSim *s, int which) {
    uint32_t T = s->table;
    int cnt = which == 0 ? s->n : s->ne;
    uint32_t *cs = which == 0 ? s->cs : s->ecs;
    uint32_t *srt = which == 0 ? s->srt : s->esrt;
    uint32_t *key = (uint32_t *)malloc(4 * ((size_t)cnt + 1));
    uint32_t *count = (uint32_t *)calloc((size_t)T + 1, 4);
    for (int i = 0; i < cnt; i++) {
        v3 q;
        if (which == 0) q = s->p[i];
        else {
            v3 p0 = s->p[s->edges[2 * i]], p1 = s->p[s->edges[2 * i + 1]];
            q = vmul(vadd(p0, p1), 0.5f);
        }
        int32_t c[3]; cell_of(q, s->cell, c);
        key[i] = hash3(c[0], c[1], c[2], T);
        count[key[i]]++;
    }
    uint32_t acc = 0;
    for (uint32_t h = 0; h < T; h++) { cs[h] = acc; acc += count[h]; }
    cs[T] = acc;
    memset(count, 0, 4 * ((size_t)T + 1));
    for (int i = 0; i < cnt; i++) { uint32_t h = key[i]; srt[cs[h] + count[h]++] = (uint32_t)i; }
    free(key); free(count);
}
static inline int32_t to_fixed(float x) { return f2i(clampf(x * 1000000.0f, -50000000.0f, 50000000.0f)); }
/* Integer accumulation is order-free; with OpenMP threads the updates are
 * atomic, so threaded and serial runs give identical bits. */
static inline void acc_add(int32_t *a, int32_t v) { __atomic_fetch_add((uint32_t *)a, (uint32_t)v, __ATOMIC_RELAXED); }
static inline void acc_inc(int32_t *a) { __atomic_fetch_add((uint32_t *)a, 1u, __ATOMIC_RELAXED); }
static inline void acc_max(int32_t *a, int32_t v) {
    int32_t cur = __atomic_load_n(a, __ATOMIC_RELAXED);
    while (v > cur && !__atomic_compare_exchange_n(a, &cur, v, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
}
static inline void acc_min(int32_t *a, int32_t v) {
    int32_t cur = __atomic_load_n(a, __ATOMIC_RELAXED);
    while (v < cur && !__atomic_compare_exchange_n(a, &cur, v, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
}
/* add_disp_atomic, shaders/self_collision.wgsl:77-85 */
static void add_disp(OSim *s, uint32_t v, v3 d) {
    int32_t *a = s->acc + (size_t)v * A_N;
    acc_add(&a[A_DX], to_fixed(d.x)); acc_add(&a[A_DY], to_fixed(d.y)); acc_add(&a[A_DZ], to_fixed(d.z));
    acc_inc(&a[A_CNT]);
}
/* add_pin_disp_atomic, shaders/self_collision.wgsl:87-95 */
static void add_pin(OSim *s, uint32_t v, v3 d) {
    int32_t *a = s->acc + (size_t)v * A_N;
    acc_add(&a[A_PDX], to_fixed(d.x)); acc_add(&a[A_PDY], to_fixed(d.y)); acc_add(&a[A_PDZ], to_fixed(d.z));
    acc_inc(&a[A_PCNT]);
}
/* add_ccd_atomic, shaders/self_collision.wgsl:97-118 and
 * shaders/self_collision_ee_direct.wgsl:97-125 (count_ee variant) */
static void add_ccd(OSim *s, uint32_t v, v3 d, int count_ee) {
    int32_t *a = s->acc + (size_t)v * A_N;
    int32_t ix = to_fixed(d.x), iy = to_fixed(d.y), iz = to_fixed(d.z);
    if (ix > 0) acc_max(&a[A_CPX], ix); else if (ix < 0) acc_min(&a[A_CNX], ix);
    if (iy > 0) acc_max(&a[A_CPY], iy); else if (iy < 0) acc_min(&a[A_CNY], iy);
    if (iz > 0) acc_max(&a[A_CPZ], iz); else if (iz < 0) acc_min(&a[A_CNZ], iz);
    if (count_ee) {
        float lf = clampf(vlen(d) * 1000000.0f, 0.0f, 2000000000.0f);
        uint32_t u = lf != lf ? 0u : (uint32_t)lf;
        if (u > 0u) acc_inc(&a[A_EEC]);
    }
}
static int th_search(const OSim *s, uint32_t a, uint32_t b, uint32_t *pos) {
    uint32_t lo = s->th_off[a], hi = s->th_off[a + 1];
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2u;
        uint32_t v = s->th_idx[mid];
        if (v == b) { *pos = mid; return 1; }
        if (v < b) lo = mid + 1u; else hi = mid;
    }
    return 0;
}
/* is_within_two_hops, shaders/self_collision.wgsl:243-264 */
static int within2(const OSim *s, uint32_t a, uint32_t b) {
    uint32_t q;
    if (a == b) return 1;
    return th_search(s, a, b, &q);
}
/* is_topologically_near_folded, shaders/self_collision.wgsl:268-293 */
static int near_folded(const OSim *s, uint32_t a, uint32_t b, float d) {
    uint32_t q;
    if (a == b) return 1;
    if (!th_search(s, a, b, &q)) return 0;
    return !(d < s->th_rest[q] * 0.5f);
}
/* is_topologically_near_folded_sq, shaders/self_collision_ee_direct.wgsl:237-262 */
static int near_folded_sq(const OSim *s, uint32_t a, uint32_t b, float d2) {
    uint32_t q;
    if (a == b) return 1;
    if (!th_search(s, a, b, &q)) return 0;
    float l0 = s->th_rest[q];
    return !(d2 < (l0 * l0) * 0.25f);
}
static inline int cell_eq(const int32_t *a, int32_t x, int32_t y, int32_t z) { return a[0] == x && a[1] == y && a[2] == z; }

/* sc_solve, shaders/self_collision.wgsl:317-681 */
/* Pair record: rows appended from the parallel loops under a lock, put in
 * canonical order when read (ocl_get_pair_lists). */
static void rec_push(uint32_t **buf, size_t *n, size_t *cap, const uint32_t *row, int width) {
    if (*n == *cap) {
        *cap = *cap ? 2 * *cap : 1024;
        *buf = (uint32_t *)realloc(*buf, *cap * (size_t)width * sizeof(uint32_t));
    }
    memcpy(*buf + *n * (size_t)width, row, (size_t)width * sizeof(uint32_t));
    (*n)++;
}
static void rec_vt(OSim *s, uint32_t i, uint32_t a, uint32_t b, uint32_t c) {
    uint32_t row[4] = {i, a, b, c};
#pragma omp critical(ocl_rec)
    rec_push(&s->rec_vt, &s->rec_vt_n, &s->rec_vt_cap, row, 4);
}
static void rec_ee(OSim *s, uint32_t ea, uint32_t eb) {
    uint32_t row[2] = {ea, eb};
#pragma omp critical(ocl_rec)
    rec_push(&s->rec_ee, &s->rec_ee_n, &s->rec_ee_cap, row, 2);
}

static void k_sc_solve(OSim *s, int untangle) {
    const float cs = s->cell;
#pragma omp parallel for schedule(dynamic, 64)
    for (uint32_t index = 0; index < (uint32_t)s->n; index++) {
        float wi = s->w[index];
        int pin_i = wi <= 0.0f;
        v3 xi = s->x[index], pi = s->p[index];
        float mli = vlen(vsub(pi, xi));
        if (pin_i && mli < EPS) continue;
        float thi = s->thick[index];
        float lli = s->local_len[index];
        int32_t cell[3]; cell_of(pi, cs, cell);
        uint32_t li = s->layer[index];
        int track = untangle && !pin_i && li > 0u;
        float best_in = 1e20f; uint32_t best_j = 0xFFFFFFFFu;
        for (int32_t cx = cell[0] - 1; cx <= cell[0] + 1; cx++)
        for (int32_t cy = cell[1] - 1; cy <= cell[1] + 1; cy++)
        for (int32_t cz = cell[2] - 1; cz <= cell[2] + 1; cz++) {
            uint32_t h = hash3(cx, cy, cz, s->table);
            for (uint32_t k = s->cs[h]; k < s->cs[h + 1]; k++) {
                uint32_t j = s->srt[k];
                if (j >= (uint32_t)s->n || j == index) continue;
                v3 pj = s->p[j];
                int32_t jc[3]; cell_of(pj, cs, jc);
                if (!cell_eq(jc, cx, cy, cz)) continue;
                v3 dvv = vsub(pi, pj);
                float d2 = vdot(dvv, dvv);
                float thj = s->thick[j], llj = s->local_len[j];
                float mind = thi + thj;
                float em = fminf(lli, llj) * 0.06f;
                float eth = fmaxf(mind, em);
                float mgd = eth + (lli + llj) * 1.3f;
                uint32_t lj = s->layer[j];
                float wj = s->w[j];
                if (track && lj < li && d2 < best_in) {
                    float ur = eth * 2.5f + llj * 1.3f;
                    if (d2 <= ur * ur && !within2(s, index, j)) { best_in = d2; best_j = j; }
                }
                if (!(d2 <= mgd * mgd)) continue;
                float dvl = sqrtf(fmaxf(d2, 0.0f));
                if (near_folded(s, index, j, dvl)) continue;
                v3 pjo = s->x[j];
                int both = wj > 0.0f;
                float eth2 = eth * eth;
                /* 1. vertex-vertex */
                if (!pin_i && (!both || index < j)) {
                    if (d2 < eth2 && d2 > EPS * EPS) {
                        int utv = 0;
                        if (untangle && li != lj) {
                            v3 ni = s->nrm[index], nj = s->nrm[j];
                            float nil = vlen(ni), njl = vlen(nj);
                            if (li > lj) {
                                if (njl > 0.5f) {
                                    v3 nju = vdiv(nj, njl);
                                    int allow = (wj <= 0.0f) || (nil <= 0.5f) || (vdot(vdiv(ni, fmaxf(nil, EPS)), nju) > 0.0f);
                                    utv = allow && (vdot(dvv, nju) < 0.0f);
                                }
                            } else if (both && nil > 0.5f) {
                                v3 niu = vdiv(ni, nil);
                                int allow = (njl <= 0.5f) || (vdot(vdiv(nj, fmaxf(njl, EPS)), niu) > 0.0f);
                                utv = allow && (vdot(vneg(dvv), niu) < 0.0f);
                            }
                        }
                        if (!utv) {
                            v3 nn = vdiv(dvv, dvl);
                            float pen = eth - dvl;
                            float ws = wi + wj;
                            if (ws > EPS) {
                                if (wj <= 0.0f) {
                                    v3 mvj = vsub(pj, pjo);
                                    add_pin(s, index, vadd(vmul(nn, pen), vmul(mvj, 0.5f)));
                                } else {
                                    v3 disp = vmul(nn, pen * 0.5f);
                                    add_disp(s, index, vmul(disp, wi / ws));
                                    add_disp(s, j, vmul(vneg(disp), wj / ws));
                                }
                            }
                        }
                    }
                }
                /* 2. vertex-triangle */
                float mli2 = vlen(vsub(pi, xi));
                float mlj = vlen(vsub(pj, pjo));
                float vtb = eth + llj * 1.3f + mli2 + mlj;
                if (!(d2 <= vtb * vtb) || within2(s, index, j)) continue;
                for (uint32_t st = s->star_off[j]; st < s->star_off[j + 1]; st++) {
                    uint32_t v0 = s->star_idx[2 * st], v1 = s->star_idx[2 * st + 1];
                    if (v0 == index || v1 == index) continue;
                    v3 pv0 = s->p[v0], pv1 = s->p[v1];
                    v3 pv0o = s->x[v0], pv1o = s->x[v1];
                    float wv0 = s->w[v0], wv1 = s->w[v1];
                    v3 d0 = vsub(pi, pv0);
                    float ll0 = s->local_len[v0];
                    float et0 = fmaxf(thi + s->thick[v0], fminf(lli, ll0) * 0.06f);
                    float b0 = et0 + ll0 * 1.3f + mli2 + vlen(vsub(pv0, pv0o));
                    int32_t c0[3]; cell_of(pv0, cs, c0);
                    int in0 = abs(c0[0] - cell[0]) <= 1 && abs(c0[1] - cell[1]) <= 1 && abs(c0[2] - cell[2]) <= 1 &&
                              (vdot(d0, d0) <= b0 * b0);
                    v3 d1 = vsub(pi, pv1);
                    float ll1 = s->local_len[v1];
                    float et1 = fmaxf(thi + s->thick[v1], fminf(lli, ll1) * 0.06f);
                    float b1 = et1 + ll1 * 1.3f + mli2 + vlen(vsub(pv1, pv1o));
                    int32_t c1[3]; cell_of(pv1, cs, c1);
                    int in1 = abs(c1[0] - cell[0]) <= 1 && abs(c1[1] - cell[1]) <= 1 && abs(c1[2] - cell[2]) <= 1 &&
                              (vdot(d1, d1) <= b1 * b1);
                    if ((in0 && j > v0) || (in1 && j > v1)) continue;
                    v3 tmove = vdiv(vadd(vadd(vsub(pj, pjo), vsub(pv0, pv0o)), vsub(pv1, pv1o)), 3.0f);
                    int tpin = (wj <= 0.0f) || (wv0 <= 0.0f) || (wv1 <= 0.0f);
                    v3 rel = vadd(xi, tmove);
                    v3 smin = vsub(vmin(rel, pi), V3(eth, eth, eth));
                    v3 smax = vadd(vmax(rel, pi), V3(eth, eth, eth));
                    v3 tmin = vmin(vmin(pj, pv0), pv1), tmax = vmax(vmax(pj, pv0), pv1);
                    if (smin.x > tmax.x || smin.y > tmax.y || smin.z > tmax.z ||
                        smax.x < tmin.x || smax.y < tmin.y || smax.z < tmin.z) continue;
                    if (within2(s, index, v0) || within2(s, index, v1)) continue;
                    if (s->rec) rec_vt(s, index, j, v0, v1);
                    v3 mv = vsub(pi, rel);
                    float msq = vdot(mv, mv);
                    float ht = 1.0f, hu = 0.0f, hv = 0.0f; int hit = 0;
                    if (msq > 1e-12f) hit = seg_tri(rel, pi, pj, pv0, pv1, &ht, &hu, &hv);
                    if (hit) {
                        v3 hp = vadd(rel, vmul(mv, ht));
                        v3 tc = vcross(vsub(pv0, pj), vsub(pv1, pj));
                        float tl = vlen(tc);
                        v3 tn = tl > 1e-12f ? vdiv(tc, tl) : V3(0.0f, 1.0f, 0.0f);
                        float hor = vdot(vsub(rel, pj), tn);
                        int utc = 0;
                        if (untangle && !pin_i && (li > lj) && tl > 1e-12f) {
                            v3 ni = s->nrm[index];
                            float nil = vlen(ni);
                            int allow = tpin || (nil <= 0.5f) || (vdot(vdiv(ni, fmaxf(nil, EPS)), tn) > 0.0f);
                            int ret = (hor < 0.0f) && (vdot(mv, tn) > 0.0f);
                            utc = allow && ret;
                        }
                        if (!utc) {
                            float ss = fabsf(hor) > 1e-6f ? hor : vdot(vneg(mv), tn);
                            v3 ns = ss >= 0.0f ? tn : vneg(tn);
                            float ho = fmaxf(vdot(vsub(rel, hp), ns), 0.0f);
                            float hs = fmaxf(ho, eth * 0.25f);
                            v3 psafe = vadd(hp, vmul(ns, hs));
                            v3 tccd = vsub(psafe, pi);
                            float pcs = fmaxf(0.0f, eth - hs);
                            if (tpin) {
                                if (!pin_i) add_ccd(s, index, vadd(tccd, vmul(ns, pcs)), 0);
                            } else if (pin_i) {
                                v3 bc = V3(clampf(1.0f - hu - hv, 0.0f, 1.0f), clampf(hu, 0.0f, 1.0f), clampf(hv, 0.0f, 1.0f));
                                float wt = bc.x * bc.x * wj + bc.y * bc.y * wv0 + bc.z * bc.z * wv1;
                                if (wt > EPS) {
                                    v3 full = vadd(tccd, vmul(ns, pcs));
                                    if (wj > 0.0f) add_ccd(s, j, vmul(vneg(full), bc.x * wj / wt), 0);
                                    if (wv0 > 0.0f) add_ccd(s, v0, vmul(vneg(full), bc.y * wv0 / wt), 0);
                                    if (wv1 > 0.0f) add_ccd(s, v1, vmul(vneg(full), bc.z * wv1 / wt), 0);
                                }
                            } else {
                                v3 bc = V3(clampf(1.0f - hu - hv, 0.0f, 1.0f), clampf(hu, 0.0f, 1.0f), clampf(hv, 0.0f, 1.0f));
                                float wt = bc.x * bc.x * wj + bc.y * bc.y * wv0 + bc.z * bc.z * wv1;
                                float wtot = wi + wt;
                                if (wtot > EPS) {
                                    add_ccd(s, index, vmul(tccd, wi / wtot), 0);
                                    if (wj > 0.0f) add_ccd(s, j, vmul(vneg(tccd), bc.x * wj / wtot), 0);
                                    if (wv0 > 0.0f) add_ccd(s, v0, vmul(vneg(tccd), bc.y * wv0 / wtot), 0);
                                    if (wv1 > 0.0f) add_ccd(s, v1, vmul(vneg(tccd), bc.z * wv1 / wtot), 0);
                                    if (pcs > EPS) {
                                        v3 tp = vmul(ns, pcs * 0.6f);
                                        add_disp(s, index, vmul(tp, wi / wtot));
                                        if (wj > 0.0f) add_disp(s, j, vmul(vneg(tp), bc.x * wj / wtot));
                                        if (wv0 > 0.0f) add_disp(s, v0, vmul(vneg(tp), bc.y * wv0 / wtot));
                                        if (wv1 > 0.0f) add_disp(s, v1, vmul(vneg(tp), bc.z * wv1 / wtot));
                                    }
                                }
                            }
                        }
                    } else {
                        int isf; v3 bary;
                        v3 cp = closest_tri(pi, pj, pv0, pv1, &isf, &bary);
                        v3 dvt = vsub(pi, cp);
                        float d2vt = vdot(dvt, dvt);
                        if (!pin_i && d2vt < eth2 && d2vt > EPS * EPS) {
                            float dvtl = sqrtf(d2vt);
                            int utv = 0;
                            if (untangle && li > lj) {
                                v3 tc = vcross(vsub(pv0, pj), vsub(pv1, pj));
                                float tl = vlen(tc);
                                if (tl > EPS) {
                                    v3 tn = vdiv(tc, tl);
                                    float hvt = vdot(dvt, tn);
                                    if (hvt < 0.0f) {
                                        v3 ni = s->nrm[index];
                                        float nil = vlen(ni);
                                        utv = tpin || (nil <= 0.5f) || (vdot(vdiv(ni, fmaxf(nil, EPS)), tn) > 0.0f);
                                    }
                                }
                            }
                            if (!utv) {
                                v3 nvt = vdiv(dvt, dvtl);
                                float pvt = eth - dvtl;
                                if (tpin) {
                                    add_pin(s, index, vadd(vmul(nvt, pvt), vmul(tmove, 0.5f)));
                                } else {
                                    float wt = bary.x * bary.x * wj + bary.y * bary.y * wv0 + bary.z * bary.z * wv1;
                                    float wtot = wi + wt;
                                    if (wtot > EPS) {
                                        v3 tp = vmul(nvt, pvt * 0.6f);
                                        add_disp(s, index, vmul(tp, wi / wtot));
                                        if (wj > 0.0f) add_disp(s, j, vmul(vneg(tp), bary.x * wj / wtot));
                                        if (wv0 > 0.0f) add_disp(s, v0, vmul(vneg(tp), bary.y * wv0 / wtot));
                                        if (wv1 > 0.0f) add_disp(s, v1, vmul(vneg(tp), bary.z * wv1 / wtot));
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
        if (track && best_j < 0x3FFFFEu) s->acc[(size_t)index * A_N + A_UT] = (int32_t)(best_j + 1u);
    }
}

/* sc_untangle, shaders/self_collision_untangle.wgsl:199-394 */
static int th_range_has(const OSim *s, uint32_t start, uint32_t end, uint32_t b) {
    if (start >= end) return 0;
    uint32_t lo = start, hi = end;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2u;
        uint32_t v = s->th_idx[mid];
        if (v == b) return 1;
        if (v < b) lo = mid + 1u; else hi = mid;
    }
    return 0;
}
static void k_untangle(OSim *s) {
#pragma omp parallel for schedule(dynamic, 64)
    for (uint32_t index = 0; index < (uint32_t)s->n; index++) {
        int32_t *ai = s->acc + (size_t)index * A_N;
        uint32_t cand = (uint32_t)ai[A_UT];
        if (cand == 0u) continue;
        ai[A_UT] = 0;
        float wi = s->w[index];
        if (wi <= 0.0f || s->layer[index] == 0u) continue;
        uint32_t j1e = cand & 0x3FFFFFu;
        if (j1e == 0u) continue;
        uint32_t j1 = j1e - 1u;
        if (j1 >= (uint32_t)s->n || j1 == index) continue;
        v3 pi = s->p[index];
        float thi = s->thick[index], lli = s->local_len[index];
        uint32_t ts = s->th_off[index], te = s->th_off[index + 1];
        uint32_t li = s->layer[index];
        uint32_t j2 = 0xFFFFFFFFu;
        float bnd = 1e20f;
        for (uint32_t a = s->adj_off[j1]; a < s->adj_off[j1 + 1]; a++) {
            uint32_t nb = s->adj_idx[a];
            if (nb < (uint32_t)s->n && nb != index && s->layer[nb] < li) {
                v3 dn = vsub(pi, s->p[nb]);
                float dns = vdot(dn, dn);
                if (dns < bnd && !th_range_has(s, ts, te, nb)) { bnd = dns; j2 = nb; }
            }
        }
        float bd2 = 1e20f, bh = 0.0f;
        uint32_t bj = 0xFFFFFFFFu, bv0 = 0, bv1 = 0;
        for (int ci = 0; ci < 2; ci++) {
            uint32_t j = ci == 0 ? j1 : j2;
            if (j == 0xFFFFFFFFu) continue;
            v3 pj = s->p[j];
            float eth = fmaxf(thi + s->thick[j], fminf(lli, s->local_len[j]) * 0.06f);
            float capt = eth * 2.5f;
            float capsq = capt * capt;
            for (uint32_t st = s->star_off[j]; st < s->star_off[j + 1]; st++) {
                uint32_t v0 = s->star_idx[2 * st], v1 = s->star_idx[2 * st + 1];
                if (v0 == index || v1 == index) continue;
                if (ci == 1 && (v0 == j1 || v1 == j1)) continue;
                v3 pv0 = s->p[v0], pv1 = s->p[v1];
                v3 tmin = vmin(vmin(pj, pv0), pv1), tmax = vmax(vmax(pj, pv0), pv1);
                v3 ad = vadd(vmax(vsub(tmin, pi), V3(0, 0, 0)), vmax(vsub(pi, tmax), V3(0, 0, 0)));
                float lim = fminf(capsq, bd2 + 1e-10f);
                if (vdot(ad, ad) >= lim) continue;
                int isf; v3 bary;
                v3 pt = closest_tri(pi, pj, pv0, pv1, &isf, &bary);
                v3 du = vsub(pi, pt);
                float dsu = vdot(du, du);
                if (dsu >= capsq) continue;
                if (bj != 0xFFFFFFFFu && dsu > bd2 + 1e-10f) continue;
                v3 tc = vcross(vsub(pv0, pj), vsub(pv1, pj));
                float tl = vlen(tc);
                if (tl <= EPS) continue;
                float hu = vdot(du, vdiv(tc, tl));
                int same = fabsf(dsu - bd2) <= 1e-10f;
                int better = (hu >= 0.0f && bh < 0.0f) || (((hu >= 0.0f) == (bh >= 0.0f)) && fabsf(hu) > fabsf(bh));
                if (bj == 0xFFFFFFFFu || dsu < bd2 - 1e-10f || (same && better)) {
                    if (th_range_has(s, ts, te, j) || th_range_has(s, ts, te, v0) || th_range_has(s, ts, te, v1)) continue;
                    bd2 = dsu; bh = hu; bj = j; bv0 = v0; bv1 = v1;
                }
            }
        }
        if (bj != 0xFFFFFFFFu && bh < 0.0f) {
            v3 upj = s->p[bj], up0 = s->p[bv0], up1 = s->p[bv1];
            float wj = s->w[bj], w0 = s->w[bv0], w1 = s->w[bv1];
            int isf; v3 bary;
            v3 pt = closest_tri(pi, upj, up0, up1, &isf, &bary);
            v3 du = vsub(pi, pt);
            float dl = vlen(du);
            v3 tc = vcross(vsub(up0, upj), vsub(up1, upj));
            float tl = vlen(tc);
            if (tl > EPS && dl > EPS) {
                v3 tn = vdiv(tc, tl);
                float hu = vdot(du, tn);
                if (hu < 0.0f) {
                    v3 ni = s->nrm[index];
                    float nil = vlen(ni);
                    int tpin = (wj <= 0.0f) || (w0 <= 0.0f) || (w1 <= 0.0f);
                    int allow = tpin || (nil <= 0.5f) || (vdot(vdiv(ni, fmaxf(nil, EPS)), tn) > 0.0f);
                    float etu = fmaxf(thi + s->thick[bj], fminf(lli, s->local_len[bj]) * 0.06f);
                    float cb = -hu / dl;
                    float rt = sqrtf(fmaxf(dl * dl - hu * hu, 0.0f));
                    float rl = fmaxf(etu * 0.5f, EPS);
                    if (allow && cb > 0.707f && rt < rl) {
                        v3 ni2 = vadd(vadd(vmul(s->nrm[bj], bary.x), vmul(s->nrm[bv0], bary.y)), vmul(s->nrm[bv1], bary.z));
                        float nl = vlen(ni2);
                        int behind = (nl <= 0.5f) || (vdot(du, ni2) < 0.0f);
                        if (behind) {
                            float cw = clampf((cb - 0.707f) / 0.2f, 0.0f, 1.0f);
                            float rw = clampf(1.0f - rt / rl, 0.0f, 1.0f);
                            float pen = fminf(etu - hu, etu * 2.0f) * cw * rw;
                            if (pen > EPS) {
                                if (tpin) add_disp(s, index, vmul(tn, pen));
                                else {
                                    float wt = bary.x * bary.x * wj + bary.y * bary.y * w0 + bary.z * bary.z * w1;
                                    float wtot = wi + wt;
                                    if (wtot > EPS) {
                                        v3 disp = vmul(tn, pen * 0.5f);
                                        add_disp(s, index, vmul(disp, wi / wtot));
                                        if (wj > 0.0f) add_disp(s, bj, vmul(vneg(disp), bary.x * wj / wtot));
                                        if (w0 > 0.0f) add_disp(s, bv0, vmul(vneg(disp), bary.y * w0 / wtot));
                                        if (w1 > 0.0f) add_disp(s, bv1, vmul(vneg(disp), bary.z * w1 / wtot));
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
    }
}

/* closest_points_segments, shaders/self_collision_ee_direct.wgsl:152-190 */
static void seg_seg(v3 p1, v3 q1, v3 p2, v3 q2, float *so, float *to) {
    v3 d1 = vsub(q1, p1), d2 = vsub(q2, p2), r = vsub(p1, p2);
    float a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
    if (a <= 1e-12f && e <= 1e-12f) { *so = 0; *to = 0; return; }
    if (a <= 1e-12f) { *so = 0; *to = clampf(f / e, 0.0f, 1.0f); return; }
    float c = vdot(d1, r);
    if (e <= 1e-12f) { *so = clampf(-c / a, 0.0f, 1.0f); *to = 0; return; }
    float b = vdot(d1, d2);
    float den = a * e - b * b;
    float s = 0.0f;
    if (den > a * e * 1e-7f) s = clampf((b * f - c * e) / den, 0.0f, 1.0f);
    float t = (b * s + f) / e;
    if (t < 0.0f) { t = 0.0f; s = clampf(-c / a, 0.0f, 1.0f); }
    else if (t > 1.0f) { t = 1.0f; s = clampf((b - c) / a, 0.0f, 1.0f); }
    *so = s; *to = t;
}
/* eval_segment_dist_sq / eval_segment_volume, :197-232 */
static float seg_eval(v3 a0o, v3 a0, v3 a1o, v3 a1, v3 b0o, v3 b0, v3 b1o, v3 b1, float tau, float *so, float *to) {
    v3 A0 = vmix(a0o, a0, tau), A1 = vmix(a1o, a1, tau), B0 = vmix(b0o, b0, tau), B1 = vmix(b1o, b1, tau);
    seg_seg(A0, A1, B0, B1, so, to);
    v3 pa = vmix(A0, A1, *so), pb = vmix(B0, B1, *to);
    v3 d = vsub(pa, pb);
    return vdot(d, d);
}
static float seg_vol(v3 a0o, v3 a0, v3 a1o, v3 a1, v3 b0o, v3 b0, v3 b1o, v3 b1, float tau) {
    v3 A0 = vmix(a0o, a0, tau), A1 = vmix(a1o, a1, tau), B0 = vmix(b0o, b0, tau), B1 = vmix(b1o, b1, tau);
    return vdot(vcross(vsub(A1, A0), vsub(B1, B0)), vsub(B0, A0));
}
/* is_outer_edge_behind_inner, :127-150 */
static int outer_behind(OSim *s, uint32_t la, uint32_t lb, uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1,
                        int afix, int bfix, v3 dab) {
    if (la == lb) return 0;
    v3 na = vadd(s->nrm[a0], s->nrm[a1]), nb = vadd(s->nrm[b0], s->nrm[b1]);
    float nal = vlen(na), nbl = vlen(nb);
    if (la > lb) {
        if (nbl <= 0.5f) return 0;
        v3 ni = vdiv(nb, nbl);
        int allow = bfix || (nal <= 0.5f) || (vdot(vdiv(na, fmaxf(nal, EPS)), ni) > 0.0f);
        return allow && (vdot(dab, ni) < 0.0f);
    }
    if (nal <= 0.5f) return 0;
    v3 ni = vdiv(na, nal);
    int allow = afix || (nbl <= 0.5f) || (vdot(vdiv(nb, fmaxf(nbl, EPS)), ni) > 0.0f);
    return allow && (vdot(vneg(dab), ni) < 0.0f);
}
static inline int ebit(const OSim *s, uint32_t e) { return (s->ebits[e >> 5] >> (e & 31u)) & 1u; }

/* sc_solve_ee, shaders/self_collision_ee_direct.wgsl:266-776 */
static void k_ee(OSim *s, int untangle) {
    const float cs = s->cell;
#pragma omp parallel for schedule(dynamic, 64)
    for (uint32_t ei = 0; ei < (uint32_t)s->ne; ei++) {
        uint32_t u0 = s->edges[2 * ei], u1 = s->edges[2 * ei + 1];
        float w_u0 = s->w[u0], w_u1 = s->w[u1];
        int pu0 = w_u0 <= 0.0f, pu1 = w_u1 <= 0.0f;
        int apin = pu0 || pu1;
        v3 p_u0 = s->p[u0], p_u1 = s->p[u1], p_u0o = s->x[u0], p_u1o = s->x[u1];
        float thu0 = s->thick[u0], thu1 = s->thick[u1];
        float mta = fmaxf(thu0, thu1);
        int bnda = ebit(s, ei);
        v3 m2 = V3(mta * 2.0f, mta * 2.0f, mta * 2.0f);
        v3 amin = vsub(vmin(vmin(p_u0, p_u1), vmin(p_u0o, p_u1o)), m2);
        v3 amax = vadd(vmax(vmax(p_u0, p_u1), vmax(p_u0o, p_u1o)), m2);
        v3 pmid = vmul(vadd(p_u0, p_u1), 0.5f);
        int32_t base[3]; cell_of(pmid, cs, base);
        uint32_t search = 0;
        int stop = 0;
        uint32_t la = s->layer[u0];
        for (int dz = -1; dz <= 1 && !stop; dz++)
        for (int dy = -1; dy <= 1 && !stop; dy++)
        for (int dx = -1; dx <= 1 && !stop; dx++) {
            int32_t nx = base[0] + dx, ny = base[1] + dy, nz = base[2] + dz;
            uint32_t h = hash3(nx, ny, nz, s->table);
            uint32_t st = s->ecs[h], en = s->ecs[h + 1];
            if (st >= en) continue;
            for (uint32_t q = 0; q < en - st; q++) {
                uint32_t eb = s->esrt[st + q];
                if (ei >= eb) continue;
                uint32_t j = s->edges[2 * eb], vj = s->edges[2 * eb + 1];
                if (j == u0 || j == u1 || vj == u0 || vj == u1) continue;
                v3 p_j = s->p[j], p_vj = s->p[vj];
                v3 bm = vmul(vadd(p_j, p_vj), 0.5f);
                int32_t bc[3]; cell_of(bm, cs, bc);
                if (!cell_eq(bc, nx, ny, nz)) continue;
                v3 p_jo = s->x[j], p_vjo = s->x[vj];
                v3 bmin = vmin(vmin(p_j, p_vj), vmin(p_jo, p_vjo));
                v3 bmax = vmax(vmax(p_j, p_vj), vmax(p_jo, p_vjo));
                if (amin.x > bmax.x || amin.y > bmax.y || amin.z > bmax.z ||
                    amax.x < bmin.x || amax.y < bmin.y || amax.z < bmin.z) continue;
                search++;
                if (search > (uint32_t)s->max_search) { stop = 1; break; }
                if (s->rec) rec_ee(s, ei, eb);
                float w_j = s->w[j], w_vj = s->w[vj];
                float thj = s->thick[j], thvj = s->thick[vj];
                uint32_t lb = s->layer[j];
                int bndb = ebit(s, eb);
                int bpair = bnda || bndb;
                int run_ccd = bpair;
                int has1 = 0;
                float s1 = 0, t1 = 0, d2c = 0, ethc = 0;
                v3 pa1 = V3(0, 0, 0), pb1 = V3(0, 0, 0), dl1 = V3(0, 0, 0);
                if (!run_ccd) {
                    seg_seg(p_u0, p_u1, p_j, p_vj, &s1, &t1);
                    pa1 = vmix(p_u0, p_u1, s1); pb1 = vmix(p_j, p_vj, t1);
                    dl1 = vsub(pa1, pb1);
                    d2c = vdot(dl1, dl1);
                    ethc = mixf(thu0, thu1, s1) + mixf(thj, thvj, t1);
                    float meg = mta + fmaxf(thj, thvj);
                    v3 dv0 = vsub(p_u0, p_u0o), dv1 = vsub(p_u1, p_u1o), dvj = vsub(p_j, p_jo), dvvj = vsub(p_vj, p_vjo);
                    v3 va = vmul(vadd(dv0, dv1), 0.5f), vb = vmul(vadd(dvj, dvvj), 0.5f);
                    float rdg = vlen(vsub(va, vb)) + 0.5f * (vlen(vsub(dv1, dv0)) + vlen(vsub(dvvj, dvj)));
                    float reach = meg + rdg;
                    if (d2c > reach * reach) continue;
                    has1 = 1;
                    v3 d0g = vsub(vmix(p_u0o, p_u1o, s1), vmix(p_jo, p_vjo, t1));
                    int g1 = rdg > ethc * 0.5f;
                    int g2 = vdot(d0g, dl1) <= 0.0f;
                    run_ccd = g1 || g2;
                }
                if (run_ccd) {
                    float msd = 1e20f, btau = 0.0f, hs = 0.125f, ms = 0, mt = 0;
                    float pv = seg_vol(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, 0.0f);
                    float zc = -1.0f;
                    for (uint32_t k = 0; k <= 8u; k++) {
                        float tk = (float)k * 0.125f;
                        float es, et;
                        float ed = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, tk, &es, &et);
                        if (ed < msd) { msd = ed; btau = tk; ms = es; mt = et; }
                        if (k > 0u) {
                            float vol = seg_vol(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, tk);
                            if (pv * vol <= 0.0f && zc < 0.0f) zc = tk - 0.0625f;
                            pv = vol;
                        }
                    }
                    if (zc >= 0.0f) {
                        float es, et;
                        float ed = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, zc, &es, &et);
                        if (ed < msd) { msd = ed; btau = zc; hs = 0.0625f; ms = es; mt = et; }
                    }
                    float tlo = fmaxf(0.0f, btau - hs), thi = fminf(1.0f, btau + hs);
                    float tstar = btau, dstar = msd, ss = ms, ts = mt;
                    for (int it = 0; it < 6; it++) {
                        float m1 = tlo + (thi - tlo) * (1.0f / 3.0f);
                        float mm2 = thi - (thi - tlo) * (1.0f / 3.0f);
                        float e1s, e1t, e2s, e2t;
                        float e1 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, m1, &e1s, &e1t);
                        float e2 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, mm2, &e2s, &e2t);
                        if (e1 < dstar) { dstar = e1; tstar = m1; ss = e1s; ts = e1t; }
                        if (e2 < dstar) { dstar = e2; tstar = mm2; ss = e2s; ts = e2t; }
                        if (e1 < e2) thi = mm2; else tlo = m1;
                    }
                    float ets = mixf(thu0, thu1, ss) + mixf(thj, thvj, ts);
                    if (dstar >= ets * ets) continue;
                    if (s->exclude_neighbors) {
                        v3 a0s = vmix(p_u0o, p_u0, tstar), a1s = vmix(p_u1o, p_u1, tstar);
                        v3 b0s = vmix(p_jo, p_j, tstar), b1s = vmix(p_vjo, p_vj, tstar);
                        v3 t0 = vsub(a0s, b0s), t1v = vsub(a0s, b1s), t2 = vsub(a1s, b0s), t3 = vsub(a1s, b1s);
                        if (near_folded_sq(s, u0, j, vdot(t0, t0)) || near_folded_sq(s, u0, vj, vdot(t1v, t1v)) ||
                            near_folded_sq(s, u1, j, vdot(t2, t2)) || near_folded_sq(s, u1, vj, vdot(t3, t3))) continue;
                    }
                    int utc = 0;
                    if (untangle && la != lb) {
                        int afx = (w_u0 == 0.0f) && (w_u1 == 0.0f);
                        int bfx = (w_j == 0.0f) && (w_vj == 0.0f);
                        v3 d0u = vmul(vsub(vadd(p_u0o, p_u1o), vadd(p_jo, p_vjo)), 0.5f);
                        v3 d1u = vmul(vsub(vadd(p_u0, p_u1), vadd(p_j, p_vj)), 0.5f);
                        v3 mu = vsub(d1u, d0u);
                        if (la > lb && !afx) {
                            v3 ni = s->nrm[j], no = s->nrm[u0];
                            int allow = bfx || (vdot(no, no) <= 0.25f);
                            utc = allow && (vdot(ni, ni) > 0.25f) && (vdot(d0u, ni) < 0.0f) && (vdot(mu, ni) > 0.0f);
                        } else if (lb > la && !bfx) {
                            v3 ni = s->nrm[u0], no = s->nrm[j];
                            int allow = afx || (vdot(no, no) <= 0.25f);
                            utc = allow && (vdot(ni, ni) > 0.25f) && (vdot(vneg(d0u), ni) < 0.0f) && (vdot(vneg(mu), ni) > 0.0f);
                        }
                    }
                    if (utc) continue;
                    float s0, t0p;
                    seg_seg(p_u0o, p_u1o, p_jo, p_vjo, &s0, &t0p);
                    v3 d0 = vsub(vmix(p_u0o, p_u1o, s0), vmix(p_jo, p_vjo, t0p));
                    float dist0 = vlen(d0);
                    if (dist0 > EPS) {
                        v3 n0 = vdiv(d0, dist0);
                        float s1b, t1b;
                        seg_seg(p_u0, p_u1, p_j, p_vj, &s1b, &t1b);
                        v3 d1 = vsub(vmix(p_u0, p_u1, s1b), vmix(p_j, p_vj, t1b));
                        float dist1 = vlen(d1);
                        v3 de = vsub(vmix(p_u0, p_u1, ss), vmix(p_j, p_vj, ts));
                        float he = vdot(de, n0);
                        int cross = (he <= 0.0f) || (vdot(d1, n0) <= 0.0f) || (bpair && dist1 >= ets && tstar < 1.0f);
                        if (he < ets && cross) {
                            float pc = ets - he;
                            int bpin = (w_j <= 0.0f) || (w_vj <= 0.0f);
                            if (apin && bpin) continue;
                            int aall = (w_u0 == 0.0f) && (w_u1 == 0.0f);
                            int ball = (w_j == 0.0f) && (w_vj == 0.0f);
                            int cpe = !(aall || ball);
                            if (bpin) {
                                v3 em = vmul(vadd(vsub(p_j, p_jo), vsub(p_vj, p_vjo)), 0.5f);
                                float a = 1.0f - ss, b = ss;
                                float den = a * a * w_u0 + b * b * w_u1;
                                if (den > EPS) {
                                    v3 pb = vadd(vmul(n0, pc), vmul(em, 0.5f));
                                    if (w_u0 > 0.0f) add_ccd(s, u0, vmul(pb, fminf((a * w_u0) / den, 2.0f)), cpe);
                                    if (w_u1 > 0.0f) add_ccd(s, u1, vmul(pb, fminf((b * w_u1) / den, 2.0f)), cpe);
                                }
                            } else if (apin) {
                                v3 em = vmul(vadd(vsub(p_u0, p_u0o), vsub(p_u1, p_u1o)), 0.5f);
                                float a = 1.0f - ts, b = ts;
                                float den = a * a * w_j + b * b * w_vj;
                                if (den > EPS) {
                                    v3 pb = vadd(vmul(vneg(n0), pc), vmul(em, 0.5f));
                                    if (w_j > 0.0f) add_ccd(s, j, vmul(pb, fminf((a * w_j) / den, 2.0f)), cpe);
                                    if (w_vj > 0.0f) add_ccd(s, vj, vmul(pb, fminf((b * w_vj) / den, 2.0f)), cpe);
                                }
                            } else {
                                float we1 = (1.0f - ss) * (1.0f - ss) * w_u0 + ss * ss * w_u1;
                                float we2 = (1.0f - ts) * (1.0f - ts) * w_j + ts * ts * w_vj;
                                float wtot = we1 + we2;
                                if (wtot > EPS) {
                                    v3 tcc = vmul(n0, pc);
                                    if (w_u0 > 0.0f) add_ccd(s, u0, vmul(tcc, (1.0f - ss) * w_u0 / wtot), 1);
                                    if (w_u1 > 0.0f) add_ccd(s, u1, vmul(tcc, ss * w_u1 / wtot), 1);
                                    if (w_j > 0.0f) add_ccd(s, j, vmul(vneg(tcc), (1.0f - ts) * w_j / wtot), 1);
                                    if (w_vj > 0.0f) add_ccd(s, vj, vmul(vneg(tcc), ts * w_vj / wtot), 1);
                                }
                            }
                            continue;
                        }
                    }
                }
                {
                    float sst, tst, d2e, eth;
                    v3 de;
                    if (has1) { sst = s1; tst = t1; de = dl1; d2e = d2c; eth = ethc; }
                    else {
                        seg_seg(p_u0, p_u1, p_j, p_vj, &sst, &tst);
                        v3 q1 = vadd(p_u0, vmul(vsub(p_u1, p_u0), sst));
                        v3 q2 = vadd(p_j, vmul(vsub(p_vj, p_j), tst));
                        de = vsub(q1, q2);
                        d2e = vdot(de, de);
                        eth = mixf(thu0, thu1, sst) + mixf(thj, thvj, tst);
                    }
                    if (d2e >= eth * eth || d2e <= EPS * EPS) continue;
                    if (s->exclude_neighbors) {
                        v3 e0 = vsub(p_u0, p_j), e1 = vsub(p_u0, p_vj), e2 = vsub(p_u1, p_j), e3 = vsub(p_u1, p_vj);
                        if (near_folded_sq(s, u0, j, vdot(e0, e0)) || near_folded_sq(s, u0, vj, vdot(e1, e1)) ||
                            near_folded_sq(s, u1, j, vdot(e2, e2)) || near_folded_sq(s, u1, vj, vdot(e3, e3))) continue;
                    }
                    float del = sqrtf(d2e);
                    int ute = 0;
                    if (untangle) {
                        int afx = (w_u0 <= 0.0f) && (w_u1 <= 0.0f);
                        int bfx = (w_j <= 0.0f) && (w_vj <= 0.0f);
                        ute = outer_behind(s, la, lb, u0, u1, j, vj, afx, bfx, de);
                    }
                    if (!ute) {
                        v3 ne = vdiv(de, del);
                        float pe = eth - del;
                        int bpin = (w_j <= 0.0f) || (w_vj <= 0.0f);
                        if (apin && bpin) continue;
                        if (bpin) {
                            v3 em = vmul(vadd(vsub(p_j, p_jo), vsub(p_vj, p_vjo)), 0.5f);
                            float a = 1.0f - sst, b = sst;
                            float den = a * a * w_u0 + b * b * w_u1;
                            if (den > EPS) {
                                v3 pb = vadd(vmul(ne, pe), vmul(em, 0.5f));
                                if (w_u0 > 0.0f) add_pin(s, u0, vmul(pb, fminf((a * w_u0) / den, 2.0f)));
                                if (w_u1 > 0.0f) add_pin(s, u1, vmul(pb, fminf((b * w_u1) / den, 2.0f)));
                            }
                        } else if (apin) {
                            v3 em = vmul(vadd(vsub(p_u0, p_u0o), vsub(p_u1, p_u1o)), 0.5f);
                            float a = 1.0f - tst, b = tst;
                            float den = a * a * w_j + b * b * w_vj;
                            if (den > EPS) {
                                v3 pb = vadd(vmul(vneg(ne), pe), vmul(em, 0.5f));
                                if (w_j > 0.0f) add_pin(s, j, vmul(pb, fminf((a * w_j) / den, 2.0f)));
                                if (w_vj > 0.0f) add_pin(s, vj, vmul(pb, fminf((b * w_vj) / den, 2.0f)));
                            }
                        } else {
                            float we1 = (1.0f - sst) * (1.0f - sst) * w_u0 + sst * sst * w_u1;
                            float we2 = (1.0f - tst) * (1.0f - tst) * w_j + tst * tst * w_vj;
                            float wtot = we1 + we2;
                            if (wtot > EPS) {
                                v3 td = vmul(ne, pe * 0.6f);
                                if (w_u0 > 0.0f) add_disp(s, u0, vmul(td, (1.0f - sst) * w_u0 / wtot));
                                if (w_u1 > 0.0f) add_disp(s, u1, vmul(td, sst * w_u1 / wtot));
                                if (w_j > 0.0f) add_disp(s, j, vmul(vneg(td), (1.0f - tst) * w_j / wtot));
                                if (w_vj > 0.0f) add_disp(s, vj, vmul(vneg(td), tst * w_vj / wtot));
                            }
                        }
                    }
                }
            }
        }
    }
}

/* sc_apply, shaders/self_collision_apply.wgsl:57-177 */
static void k_apply(OSim *s) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->n; i++) {
        int32_t *a = s->acc + (size_t)i * A_N;
        int pinned = s->w[i] <= 0.0f;
        v3 fd = V3(0, 0, 0);
        uint32_t cnt = (uint32_t)a[A_CNT];
        if (cnt > 0u) {
            if (!pinned) {
                v3 tdp = vmul(V3((float)a[A_DX], (float)a[A_DY], (float)a[A_DZ]), 1.0f / 1000000.0f);
                v3 ed = vdiv(tdp, fmaxf(1.0f, sqrtf((float)cnt)));
                if (s->enable_relief) ed = vmul(ed, s->relief);
                float pl = vlen(ed);
                float ratio = s->max_disp_ratio > 0.0f ? s->max_disp_ratio : 0.50f;
                float ms = fminf(s->local_len[i] * ratio, 0.10f);
                if (pl > ms && pl > EPS) ed = vmul(vdiv(ed, pl), ms);
                fd = vadd(fd, ed);
            }
            a[A_DX] = a[A_DY] = a[A_DZ] = 0; a[A_CNT] = 0;
        }
        uint32_t pc = (uint32_t)a[A_PCNT];
        v3 avg = V3(0, 0, 0);
        if (pc > 0u) {
            if (!pinned)
                avg = vdiv(vmul(V3((float)a[A_PDX], (float)a[A_PDY], (float)a[A_PDZ]), 1.0f / 1000000.0f), (float)pc);
            a[A_PDX] = a[A_PDY] = a[A_PDZ] = 0; a[A_PCNT] = 0;
        }
        int32_t rpx = a[A_CPX], rpy = a[A_CPY], rpz = a[A_CPZ], rnx = a[A_CNX], rny = a[A_CNY], rnz = a[A_CNZ];
        a[A_CPX] = a[A_CPY] = a[A_CPZ] = a[A_CNX] = a[A_CNY] = a[A_CNZ] = 0;
        uint32_t eec = (uint32_t)a[A_EEC];
        a[A_EEC] = 0; a[A_UT] = 0;
        if (!pinned) {
            v3 cp = vmul(V3((float)rpx, (float)rpy, (float)rpz), 1.0f / 1000000.0f);
            v3 cn = vmul(V3((float)rnx, (float)rny, (float)rnz), 1.0f / 1000000.0f);
            v3 env = vadd(cp, cn);
            if (eec >= 4u) {
                float sc = fmaxf(0.5f, sqrtf(3.0f / (float)eec));
                env = vmul(env, sc);
            }
            v3 z = V3(0, 0, 0);
            v3 hp = vmax(vmax(env, z), vmax(avg, z));
            v3 hn = vmin(vmin(env, z), vmin(avg, z));
            fd = vadd(fd, vadd(hp, hn));
        }
        if (vlen(fd) > EPS) s->p[i] = vadd(s->p[i], fd);
    }
}

/* ------------------------------------------------------------------ */
/* Contact-pair cache (self-collision algorithm 1, "Active Pair        */
/* Caching"): broad phase once per frame into per-vertex top-K slots,  */
/* narrow phase per substep over the slots.                             */
/* ------------------------------------------------------------------ */
/* |cell_a - cell_b| > 1 on one axis, 32-bit wrap and abs(INT_MIN) = INT_MIN */
static int pc_far_axis(int32_t a, int32_t b) {
    uint32_t d = (uint32_t)a - (uint32_t)b;
    uint32_t ad = ((int32_t)d < 0) ? 0u - d : d;
    return (int32_t)ad > 1;
}
/* velocity horizon, collect_pairs.wgsl:328-330 */
static float pc_horizon(const OSim *s, float dt, uint32_t i) {
    return fminf(vlen(s->v[i]) * dt * s->pair_hscale, s->pair_maxh);
}
/* can_ee_anchor_reach, shaders/self_collision_collect_pairs.wgsl:262-283 */
static int pc_anchor_reach(const OSim *s, float dt, uint32_t u, uint32_t w) {
    if (s->w[u] <= 0.0f) return 0;
    int32_t cu[3], cw[3];
    cell_of(s->p[u], s->cell, cu);
    cell_of(s->p[w], s->cell, cw);
    if (pc_far_axis(cu[0], cw[0]) || pc_far_axis(cu[1], cw[1]) || pc_far_axis(cu[2], cw[2])) return 0;
    v3 d = vsub(s->p[u], s->p[w]);
    float d2 = vdot(d, d);
    float mf = (float)s->pair_margin_mode;
    float hu = pc_horizon(s, dt, u) * mf, hw = pc_horizon(s, dt, w) * mf;
    float b = s->thick[u] + s->thick[w] + (s->local_len[u] + s->local_len[w]) * 1.3f + s->pair_safety + hu + hw;
    if (d2 > b * b) return 0;
    if ((s->island[u] == s->island[w]) && s->exclude_neighbors) {
        float dist = sqrtf(fmaxf(d2, 0.0f));
        if (near_folded(s, u, w, dist)) return 0;
    }
    return 1;
}
/* is_smaller_anchor_reachable, :286-292 */
static int pc_smaller_anchor(const OSim *s, float dt, uint32_t u, uint32_t w, uint32_t cu, uint32_t cw) {
    if (u > cu || (u == cu && w >= cw)) return 0;
    return pc_anchor_reach(s, dt, u, w);
}
typedef struct { uint32_t n, eval, drop; float d[8]; uint32_t k[8][3]; } OTopK;
/* top-K insertion with duplicate rejection, :428-475 and :558-604 */
static void topk_insert(OTopK *t, uint32_t quota, float d, uint32_t k0, uint32_t k1, uint32_t k2) {
    for (uint32_t q = 0; q < 8u; q++) {
        if (q >= t->n) break;
        if (t->k[q][0] == k0 && t->k[q][1] == k1 && t->k[q][2] == k2) return;
    }
    t->eval++;
    uint32_t pos = t->n;
    for (uint32_t q = 0; q < 8u; q++) {
        if (q < t->n) {
            const uint32_t *e = t->k[q];
            int tie = (d == t->d[q]) && (k0 < e[0] || (k0 == e[0] && (k1 < e[1] || (k1 == e[1] && k2 < e[2]))));
            if (d < t->d[q] || tie) { pos = q; break; }
        }
    }
    if (pos < quota) {
        uint32_t up = t->n < quota - 1u ? t->n : quota - 1u;
        for (uint32_t q = up; q > pos; q--) {
            t->d[q] = t->d[q - 1];
            t->k[q][0] = t->k[q - 1][0]; t->k[q][1] = t->k[q - 1][1]; t->k[q][2] = t->k[q - 1][2];
        }
        t->d[pos] = d;
        t->k[pos][0] = k0; t->k[pos][1] = k1; t->k[pos][2] = k2;
        if (t->n < quota) t->n++;
    } else {
        t->drop++;
    }
}
/* pair_collect, shaders/self_collision_collect_pairs.wgsl:293-661 */
static void k_pair_collect(OSim *s, float dt) {
    const float cs = s->cell;
    const uint32_t n = (uint32_t)s->n;
    const uint32_t qvt = s->pair_qvt < 1u ? 1u : (s->pair_qvt > 8u ? 8u : s->pair_qvt);
    const uint32_t qee = s->pair_qee < 1u ? 1u : (s->pair_qee > 8u ? 8u : s->pair_qee);
    uint64_t c_vt = 0, c_ee = 0, c_vtd = 0, c_eed = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : c_vt, c_ee, c_vtd, c_eed)
    for (uint32_t index = 0; index < n; index++) {
        int pin_i = s->w[index] <= 0.0f;
        v3 p_i = s->p[index];
        float ll_i = s->local_len[index];
        int32_t base[3];
        cell_of(p_i, cs, base);
        OTopK vt, ee;
        memset(&vt, 0, sizeof vt);
        memset(&ee, 0, sizeof ee);
        float margin = s->pair_safety;
        float h_i = pc_horizon(s, dt, index);
        for (int gx = -1; gx <= 1; gx++)
            for (int gy = -1; gy <= 1; gy++)
                for (int gz = -1; gz <= 1; gz++) {
                    int32_t cx = base[0] + gx, cy = base[1] + gy, cz = base[2] + gz;
                    uint32_t h = hash3(cx, cy, cz, s->table);
                    uint32_t st = s->cs[h], en = s->cs[h + 1];
                    if (st >= en) continue;
                    for (uint32_t k = st; k < en; k++) {
                        uint32_t j = s->srt[k];
                        if (j >= n || j == index) continue;
                        v3 p_j = s->p[j];
                        int32_t jc[3];
                        cell_of(p_j, cs, jc);
                        if (!cell_eq(jc, cx, cy, cz)) continue;
                        int pin_j = s->w[j] <= 0.0f;
                        if (!(pin_i && pin_j)) {
                            float mf = (float)s->pair_margin_mode;
                            float h_j = pc_horizon(s, dt, j) * mf;
                            float h_ie = h_i * mf;
                            v3 dvv = vsub(p_i, p_j);
                            float d2vv = vdot(dvv, dvv);
                            float eth = s->thick[index] + s->thick[j];
                            float ll_j = s->local_len[j];
                            float broad = eth + (ll_i + ll_j) * 1.3f + margin + h_ie + h_j;
                            if (d2vv <= broad * broad) {
                                int same_island = s->island[index] == s->island[j];
                                float dvvl = sqrtf(fmaxf(d2vv, 0.0f));
                                int near_topo = same_island && s->exclude_neighbors && near_folded(s, index, j, dvvl);
                                if (!near_topo) {
                                    /* 1. vertex-triangle */
                                    float vtb = eth + ll_j * 1.3f + margin + h_ie + h_j;
                                    int near2 = s->exclude_neighbors && within2(s, index, j);
                                    if (d2vv <= vtb * vtb && !near2) {
                                        uint32_t ss = s->star_off[j], se = s->star_off[j + 1];
                                        if (ss < se) {
                                            uint32_t ns = se - ss < 8u ? se - ss : 8u;
                                            for (uint32_t t = 0; t < ns; t++) {
                                                uint32_t v0 = s->star_idx[2 * (ss + t)], v1 = s->star_idx[2 * (ss + t) + 1];
                                                if (index != v0 && index != v1 && v0 < n && v1 < n) {
                                                    uint32_t c0 = j, c1 = v0, c2 = v1;
                                                    if (v0 < j && v0 < v1) { c0 = v0; c1 = v1; c2 = j; }
                                                    else if (v1 < j && v1 < v0) { c0 = v1; c1 = j; c2 = v0; }
                                                    int isf; v3 bary;
                                                    v3 cp = closest_tri(p_i, s->p[c0], s->p[c1], s->p[c2], &isf, &bary);
                                                    v3 dvt = vsub(p_i, cp);
                                                    float d2vt = vdot(dvt, dvt);
                                                    float chk = eth + margin + h_ie + h_j;
                                                    if (d2vt < chk * chk) {
                                                        if (s->exclude_neighbors) {
                                                            if (within2(s, index, v0) || within2(s, index, v1)) continue;
                                                        }
                                                        topk_insert(&vt, qvt, d2vt, c0, c1, c2);
                                                    }
                                                }
                                            }
                                        }
                                    }
                                    /* 2. edge-edge */
                                    float eeb = eth + (ll_i + ll_j) * 1.3f + margin + h_ie + h_j;
                                    if (d2vv <= eeb * eeb) {
                                        uint32_t ai0 = s->adj_off[index], ai1 = s->adj_off[index + 1];
                                        uint32_t aj0 = s->adj_off[j], aj1 = s->adj_off[j + 1];
                                        if (ai0 < ai1 && aj0 < aj1) {
                                            uint32_t nei = ai1 - ai0 < 8u ? ai1 - ai0 : 8u;
                                            uint32_t nej = aj1 - aj0 < 8u ? aj1 - aj0 : 8u;
                                            for (uint32_t e1 = 0; e1 < nei; e1++) {
                                                uint32_t ui = s->adj_idx[ai0 + e1];
                                                if (ui >= n) continue;
                                                v3 p_ui = s->p[ui];
                                                float ll_ui = s->local_len[ui];
                                                v3 li = vsub(p_ui, p_i);
                                                float lsi = vdot(li, li);
                                                float mli = (ll_i + ll_ui) * 1.5f;
                                                if (lsi > mli * mli || lsi <= 1e-12f) continue;
                                                for (uint32_t e2 = 0; e2 < nej; e2++) {
                                                    uint32_t vj = s->adj_idx[aj0 + e2];
                                                    if (vj >= n) continue;
                                                    if (ui != j && ui != vj && index != vj) {
                                                        uint32_t cj = j < vj ? j : vj, cvj = j < vj ? vj : j;
                                                        int smaller = pc_smaller_anchor(s, dt, index, vj, index, j) ||
                                                                      pc_smaller_anchor(s, dt, ui, j, index, j) ||
                                                                      pc_smaller_anchor(s, dt, ui, vj, index, j) ||
                                                                      pc_smaller_anchor(s, dt, j, index, index, j) ||
                                                                      pc_smaller_anchor(s, dt, j, ui, index, j) ||
                                                                      pc_smaller_anchor(s, dt, vj, index, index, j) ||
                                                                      pc_smaller_anchor(s, dt, vj, ui, index, j);
                                                        if (!pin_i && !smaller) {
                                                            v3 p_vj = s->p[vj];
                                                            float ll_vj = s->local_len[vj];
                                                            v3 lj = vsub(p_vj, p_j);
                                                            float lsj = vdot(lj, lj);
                                                            float mlj = (ll_j + ll_vj) * 1.5f;
                                                            if (lsj > mlj * mlj || lsj <= 1e-12f) continue;
                                                            v3 pcj = j < vj ? p_j : p_vj, pcvj = j < vj ? p_vj : p_j;
                                                            float sp, tp;
                                                            seg_seg(p_i, p_ui, pcj, pcvj, &sp, &tp);
                                                            v3 pt1 = vadd(p_i, vmul(vsub(p_ui, p_i), sp));
                                                            v3 pt2 = vadd(pcj, vmul(vsub(pcvj, pcj), tp));
                                                            v3 dee = vsub(pt1, pt2);
                                                            float d2ee = vdot(dee, dee);
                                                            float chk = eth + margin + h_ie + h_j;
                                                            if (d2ee < chk * chk && d2ee > EPS * EPS) {
                                                                if (s->exclude_neighbors) {
                                                                    if (near_folded(s, index, vj, vlen(vsub(p_i, p_vj))) ||
                                                                        near_folded(s, ui, j, vlen(vsub(p_ui, p_j))) ||
                                                                        near_folded(s, ui, vj, vlen(vsub(p_ui, p_vj))))
                                                                        continue;
                                                                }
                                                                topk_insert(&ee, qee, d2ee, ui, cj, cvj);
                                                            }
                                                        }
                                                    }
                                                }
                                            }
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
        uint32_t *bv = s->pvt + (size_t)index * qvt * 4;
        for (uint32_t q = 0; q < qvt; q++) {
            if (q < vt.n) { bv[4 * q] = index; bv[4 * q + 1] = vt.k[q][0]; bv[4 * q + 2] = vt.k[q][1]; bv[4 * q + 3] = vt.k[q][2]; }
            else { bv[4 * q] = 0xFFFFFFFFu; bv[4 * q + 1] = bv[4 * q + 2] = bv[4 * q + 3] = 0u; }
        }
        uint32_t *be = s->pee + (size_t)index * qee * 4;
        for (uint32_t q = 0; q < qee; q++) {
            if (q < ee.n) { be[4 * q] = index; be[4 * q + 1] = ee.k[q][0]; be[4 * q + 2] = ee.k[q][1]; be[4 * q + 3] = ee.k[q][2]; }
            else { be[4 * q] = 0xFFFFFFFFu; be[4 * q + 1] = be[4 * q + 2] = be[4 * q + 3] = 0u; }
        }
        c_vt += vt.eval; c_vtd += vt.drop; c_ee += ee.eval; c_eed += ee.drop;
    }
    s->pcnt[0] += (uint32_t)c_vt; s->pcnt[1] += (uint32_t)c_ee;
    s->pcnt[2] += (uint32_t)c_vtd; s->pcnt[3] += (uint32_t)c_eed;
}
static inline void acc_umax(int32_t *a, uint32_t v) {
    uint32_t *u = (uint32_t *)a;
    uint32_t cur = __atomic_load_n(u, __ATOMIC_RELAXED);
    while (v > cur && !__atomic_compare_exchange_n(u, &cur, v, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
}
/* record_untangle_cand, shaders/self_collision_solve_vt.wgsl:99-108 */
static void pc_untangle_cand(OSim *s, uint32_t vi, uint32_t j, float dist, float cap) {
    if (vi >= (uint32_t)s->n || j >= 0x3FFFFEu || dist >= cap) return;
    float ratio = clampf(dist / fmaxf(cap, EPS), 0.0f, 1.0f);
    uint32_t rank = 1023u - (uint32_t)(ratio * 1023.0f);
    uint32_t packed = (rank << 22) | ((j + 1u) & 0x3FFFFFu);
    acc_umax(&s->acc[(size_t)vi * A_N + A_UT], packed);
}
/* pair_vt, shaders/self_collision_solve_vt.wgsl:227-414 */
static void k_pair_vt(OSim *s, int untangle) {
    const uint32_t n = (uint32_t)s->n;
    const uint32_t slots = n * s->pair_qvt;
#pragma omp parallel for schedule(dynamic, 256)
    for (uint32_t slot = 0; slot < slots; slot++) {
        const uint32_t *pr = s->pvt + 4 * (size_t)slot;
        if (pr[0] == 0xFFFFFFFFu) continue;
        uint32_t index = pr[0], j = pr[1], v0 = pr[2], v1 = pr[3];
        if (index >= n || j >= n || v0 >= n || v1 >= n) continue;
        if (index == j || index == v0 || index == v1 || v0 == v1 || j == v0 || j == v1) continue;
        int pin_i = s->w[index] <= 0.0f;
        v3 p_i = s->p[index], xo = s->x[index];
        v3 p_j = s->p[j], p_v0 = s->p[v0], p_v1 = s->p[v1];
        v3 p_jo = s->x[j], p_v0o = s->x[v0], p_v1o = s->x[v1];
        float w_i = s->w[index], w_j = s->w[j], w_v0 = s->w[v0], w_v1 = s->w[v1];
        float eth = s->thick[index] + s->thick[j];
        v3 tmove = vdiv(vadd(vadd(vsub(p_j, p_jo), vsub(p_v0, p_v0o)), vsub(p_v1, p_v1o)), 3.0f);
        int tpin = (w_j <= 0.0f) || (w_v0 <= 0.0f) || (w_v1 <= 0.0f);
        int upair = untangle && !pin_i && (s->layer[index] > s->layer[j]);
        v3 niraw = upair ? s->nrm[index] : V3(0, 0, 0);
        float nil = vlen(niraw);
        v3 niu = nil > 0.5f ? vdiv(niraw, fmaxf(nil, EPS)) : V3(0, 0, 0);
        v3 rel = vadd(xo, tmove);
        float ht = 0.0f, hu = 0.0f, hv = 0.0f;
        if (seg_tri(rel, p_i, p_j, p_v0, p_v1, &ht, &hu, &hv)) {
            v3 mv = vsub(p_i, rel);
            v3 hp = vadd(rel, vmul(mv, ht));
            v3 tc = vcross(vsub(p_v0, p_j), vsub(p_v1, p_j));
            float tl = vlen(tc);
            v3 tn = tl > 1e-12f ? vdiv(tc, tl) : V3(0, 1, 0);
            float hor = vdot(vsub(rel, p_j), tn);
            int utc = 0;
            if (upair && tl > 1e-12f) {
                int allow = tpin || (nil <= 0.5f) || (vdot(niu, tn) > 0.0f);
                int ret = (hor < 0.0f) && (vdot(mv, tn) > 0.0f);
                utc = allow && ret;
            }
            if (!utc) {
                float sgn = fabsf(hor) > 1e-6f ? hor : vdot(vneg(mv), tn);
                v3 ns = sgn >= 0.0f ? tn : vneg(tn);
                float ho = fmaxf(vdot(vsub(rel, hp), ns), 0.0f);
                float hs = fmaxf(ho, eth * 0.25f);
                v3 psafe = vadd(hp, vmul(ns, hs));
                v3 tccd = vsub(psafe, p_i);
                float pcs = fmaxf(0.0f, eth - hs);
                if (tpin) {
                    if (!pin_i) add_ccd(s, index, vadd(tccd, vmul(ns, pcs)), 0);
                } else if (pin_i) {
                    v3 bc = V3(clampf(1.0f - hu - hv, 0.0f, 1.0f), clampf(hu, 0.0f, 1.0f), clampf(hv, 0.0f, 1.0f));
                    float wt = bc.x * bc.x * w_j + bc.y * bc.y * w_v0 + bc.z * bc.z * w_v1;
                    if (wt > EPS) {
                        v3 full = vadd(tccd, vmul(ns, pcs));
                        if (w_j > 0.0f) add_ccd(s, j, vmul(vneg(full), bc.x * w_j / wt), 0);
                        if (w_v0 > 0.0f) add_ccd(s, v0, vmul(vneg(full), bc.y * w_v0 / wt), 0);
                        if (w_v1 > 0.0f) add_ccd(s, v1, vmul(vneg(full), bc.z * w_v1 / wt), 0);
                    }
                } else {
                    v3 bc = V3(clampf(1.0f - hu - hv, 0.0f, 1.0f), clampf(hu, 0.0f, 1.0f), clampf(hv, 0.0f, 1.0f));
                    float wt = bc.x * bc.x * w_j + bc.y * bc.y * w_v0 + bc.z * bc.z * w_v1;
                    float wtot = w_i + wt;
                    if (wtot > EPS) {
                        add_ccd(s, index, vmul(tccd, w_i / wtot), 0);
                        if (w_j > 0.0f) add_ccd(s, j, vmul(vneg(tccd), bc.x * w_j / wtot), 0);
                        if (w_v0 > 0.0f) add_ccd(s, v0, vmul(vneg(tccd), bc.y * w_v0 / wtot), 0);
                        if (w_v1 > 0.0f) add_ccd(s, v1, vmul(vneg(tccd), bc.z * w_v1 / wtot), 0);
                        if (pcs > EPS) {
                            v3 tp = vmul(ns, pcs * 0.6f);
                            add_disp(s, index, vmul(tp, w_i / wtot));
                            if (w_j > 0.0f) add_disp(s, j, vmul(vneg(tp), bc.x * w_j / wtot));
                            if (w_v0 > 0.0f) add_disp(s, v0, vmul(vneg(tp), bc.y * w_v0 / wtot));
                            if (w_v1 > 0.0f) add_disp(s, v1, vmul(vneg(tp), bc.z * w_v1 / wtot));
                        }
                    }
                }
            } else {
                pc_untangle_cand(s, index, j, vlen(vsub(p_i, hp)), eth * 2.5f);
            }
        } else {
            int isf; v3 bary;
            v3 cp = closest_tri(p_i, p_j, p_v0, p_v1, &isf, &bary);
            v3 dvt = vsub(p_i, cp);
            float dist = vlen(dvt);
            v3 tc = vcross(vsub(p_v0, p_j), vsub(p_v1, p_j));
            float tl = vlen(tc);
            v3 tn = tl > EPS ? vdiv(tc, fmaxf(tl, EPS)) : V3(0, 0, 0);
            float hvt = tl > EPS ? vdot(dvt, tn) : 0.0f;
            int allow = tpin || (nil <= 0.5f) || (vdot(niu, tn) > 0.0f);
            int utv = upair && (tl > EPS) && allow && (hvt < 0.0f);
            if (utv) pc_untangle_cand(s, index, j, dist, eth * 2.5f);
            if (!pin_i && !utv && dist < eth && dist > EPS) {
                v3 nvt = vdiv(dvt, dist);
                float pen = eth - dist;
                if (tpin) {
                    add_pin(s, index, vadd(vmul(nvt, pen), vmul(tmove, 0.5f)));
                } else {
                    float wt = bary.x * bary.x * w_j + bary.y * bary.y * w_v0 + bary.z * bary.z * w_v1;
                    float wtot = w_i + wt;
                    if (wtot > EPS) {
                        v3 tp = vmul(nvt, pen * 0.6f);
                        add_disp(s, index, vmul(tp, w_i / wtot));
                        if (w_j > 0.0f) add_disp(s, j, vmul(vneg(tp), bary.x * w_j / wtot));
                        if (w_v0 > 0.0f) add_disp(s, v0, vmul(vneg(tp), bary.y * w_v0 / wtot));
                        if (w_v1 > 0.0f) add_disp(s, v1, vmul(vneg(tp), bary.z * w_v1 / wtot));
                    }
                }
            }
        }
    }
}
/* pair_ee, shaders/self_collision_solve_ee.wgsl:230-589 */
static void k_pair_ee(OSim *s, int untangle) {
    const uint32_t n = (uint32_t)s->n;
    const uint32_t slots = n * s->pair_qee;
#pragma omp parallel for schedule(dynamic, 256)
    for (uint32_t slot = 0; slot < slots; slot++) {
        const uint32_t *pr = s->pee + 4 * (size_t)slot;
        if (pr[0] == 0xFFFFFFFFu) continue;
        uint32_t u0 = pr[0], u1 = pr[1], j = pr[2], vj = pr[3];
        if (u0 >= n || u1 >= n || j >= n || vj >= n) continue;
        if (u0 == u1 || j == vj || u0 == j || u0 == vj || u1 == j || u1 == vj) continue;
        float w_u0 = s->w[u0], w_u1 = s->w[u1], w_j = s->w[j], w_vj = s->w[vj];
        int apin = (w_u0 <= 0.0f) || (w_u1 <= 0.0f);
        int bpin = (w_j <= 0.0f) || (w_vj <= 0.0f);
        if (apin && bpin) continue;
        v3 p_u0 = s->p[u0], p_u1 = s->p[u1], p_j = s->p[j], p_vj = s->p[vj];
        v3 p_u0o = s->x[u0], p_u1o = s->x[u1], p_jo = s->x[j], p_vjo = s->x[vj];
        float thu0 = s->thick[u0], thu1 = s->thick[u1], thj = s->thick[j], thvj = s->thick[vj];
        float s1, t1;
        seg_seg(p_u0, p_u1, p_j, p_vj, &s1, &t1);
        v3 d1c = vsub(vmix(p_u0, p_u1, s1), vmix(p_j, p_vj, t1));
        float d2c = vdot(d1c, d1c);
        float eth = mixf(thu0, thu1, s1) + mixf(thj, thvj, t1);
        float meth = fmaxf(thu0, thu1) + fmaxf(thj, thvj);
        v3 dv0 = vsub(p_u0, p_u0o), dv1 = vsub(p_u1, p_u1o), dvj = vsub(p_j, p_jo), dvvj = vsub(p_vj, p_vjo);
        v3 va = vmul(vadd(dv0, dv1), 0.5f), vb = vmul(vadd(dvj, dvvj), 0.5f);
        float rd = vlen(vsub(va, vb)) + 0.5f * (vlen(vsub(dv1, dv0)) + vlen(vsub(dvvj, dvj)));
        float reach = meth + rd;
        if (d2c > reach * reach) continue;
        v3 d0g = vsub(vmix(p_u0o, p_u1o, s1), vmix(p_jo, p_vjo, t1));
        int run_ccd = (rd > eth * 0.5f) || (vdot(d0g, d1c) <= 0.0f);
        uint32_t la = s->layer[u0], lb = s->layer[j];
        if (run_ccd) {
            float msd = 1e20f, btau = 0.0f, hs = 0.125f, ms = 0, mt = 0;
            float pv = seg_vol(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, 0.0f);
            float zc = -1.0f;
            for (uint32_t k = 0; k <= 8u; k++) {
                float tk = (float)k * 0.125f;
                float es, et;
                float ed = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, tk, &es, &et);
                if (ed < msd) { msd = ed; btau = tk; ms = es; mt = et; }
                if (k > 0u) {
                    float vol = seg_vol(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, tk);
                    if (pv * vol <= 0.0f && zc < 0.0f) zc = tk - 0.0625f;
                    pv = vol;
                }
            }
            if (zc >= 0.0f) {
                float es, et;
                float ed = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, zc, &es, &et);
                if (ed < msd) { msd = ed; btau = zc; hs = 0.0625f; ms = es; mt = et; }
            }
            float tlo = fmaxf(0.0f, btau - hs), thi = fminf(1.0f, btau + hs);
            float dstar = msd, ss = ms, ts = mt;
            for (int it = 0; it < 6; it++) {
                float m1 = tlo + (thi - tlo) * (1.0f / 3.0f);
                float mm2 = thi - (thi - tlo) * (1.0f / 3.0f);
                float e1s, e1t, e2s, e2t;
                float e1 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, m1, &e1s, &e1t);
                float e2 = seg_eval(p_u0o, p_u0, p_u1o, p_u1, p_jo, p_j, p_vjo, p_vj, mm2, &e2s, &e2t);
                if (e1 < dstar) { dstar = e1; ss = e1s; ts = e1t; }
                if (e2 < dstar) { dstar = e2; ss = e2s; ts = e2t; }
                if (e1 < e2) thi = mm2; else tlo = m1;
            }
            float ets = mixf(thu0, thu1, ss) + mixf(thj, thvj, ts);
            if (dstar >= ets * ets) continue;
            int utc = 0;
            if (untangle && la != lb) {
                int afx = (w_u0 == 0.0f) && (w_u1 == 0.0f);
                int bfx = (w_j == 0.0f) && (w_vj == 0.0f);
                v3 d0u = vmul(vsub(vadd(p_u0o, p_u1o), vadd(p_jo, p_vjo)), 0.5f);
                v3 d1u = vmul(vsub(vadd(p_u0, p_u1), vadd(p_j, p_vj)), 0.5f);
                v3 mu = vsub(d1u, d0u);
                if (la > lb && !afx) {
                    v3 ni = s->nrm[j], no = s->nrm[u0];
                    int allow = bfx || (vdot(no, no) <= 0.25f);
                    utc = allow && (vdot(ni, ni) > 0.25f) && (vdot(d0u, ni) < 0.0f) && (vdot(mu, ni) > 0.0f);
                } else if (lb > la && !bfx) {
                    v3 ni = s->nrm[u0], no = s->nrm[j];
                    int allow = afx || (vdot(no, no) <= 0.25f);
                    utc = allow && (vdot(ni, ni) > 0.25f) && (vdot(vneg(d0u), ni) < 0.0f) && (vdot(vneg(mu), ni) > 0.0f);
                }
            }
            if (utc) continue;
            float s0, t0p;
            seg_seg(p_u0o, p_u1o, p_jo, p_vjo, &s0, &t0p);
            v3 d0 = vsub(vmix(p_u0o, p_u1o, s0), vmix(p_jo, p_vjo, t0p));
            float dist0 = vlen(d0);
            if (dist0 > EPS) {
                v3 n0 = vdiv(d0, dist0);
                v3 de = vsub(vmix(p_u0, p_u1, ss), vmix(p_j, p_vj, ts));
                float he = vdot(de, n0);
                int crossed = (he <= 0.0f) || (vdot(d1c, n0) <= 0.0f);
                if (he < ets && crossed) {
                    float pc = ets - he;
                    int aall = (w_u0 == 0.0f) && (w_u1 == 0.0f);
                    int ball = (w_j == 0.0f) && (w_vj == 0.0f);
                    int cpe = !(aall || ball);
                    if (bpin) {
                        v3 em = vmul(vadd(vsub(p_j, p_jo), vsub(p_vj, p_vjo)), 0.5f);
                        float a = 1.0f - ss, b = ss;
                        float den = a * a * w_u0 + b * b * w_u1;
                        if (den > EPS) {
                            v3 pb = vadd(vmul(n0, pc), vmul(em, 0.5f));
                            if (w_u0 > 0.0f) add_ccd(s, u0, vmul(pb, fminf((a * w_u0) / den, 2.0f)), cpe);
                            if (w_u1 > 0.0f) add_ccd(s, u1, vmul(pb, fminf((b * w_u1) / den, 2.0f)), cpe);
                        }
                    } else if (apin) {
                        v3 em = vmul(vadd(vsub(p_u0, p_u0o), vsub(p_u1, p_u1o)), 0.5f);
                        float a = 1.0f - ts, b = ts;
                        float den = a * a * w_j + b * b * w_vj;
                        if (den > EPS) {
                            v3 pb = vadd(vmul(vneg(n0), pc), vmul(em, 0.5f));
                            if (w_j > 0.0f) add_ccd(s, j, vmul(pb, fminf((a * w_j) / den, 2.0f)), cpe);
                            if (w_vj > 0.0f) add_ccd(s, vj, vmul(pb, fminf((b * w_vj) / den, 2.0f)), cpe);
                        }
                    } else {
                        float we1 = (1.0f - ss) * (1.0f - ss) * w_u0 + ss * ss * w_u1;
                        float we2 = (1.0f - ts) * (1.0f - ts) * w_j + ts * ts * w_vj;
                        float wtot = we1 + we2;
                        if (wtot > EPS) {
                            v3 tcc = vmul(n0, pc);
                            if (w_u0 > 0.0f) add_ccd(s, u0, vmul(tcc, (1.0f - ss) * w_u0 / wtot), 1);
                            if (w_u1 > 0.0f) add_ccd(s, u1, vmul(tcc, ss * w_u1 / wtot), 1);
                            if (w_j > 0.0f) add_ccd(s, j, vmul(vneg(tcc), (1.0f - ts) * w_j / wtot), 1);
                            if (w_vj > 0.0f) add_ccd(s, vj, vmul(vneg(tcc), ts * w_vj / wtot), 1);
                        }
                    }
                    continue;
                }
            }
        }
        /* discrete segment repulsion */
        if (d2c >= eth * eth || d2c <= EPS * EPS) continue;
        float del = sqrtf(d2c);
        int ute = 0;
        if (untangle) {
            int afx = (w_u0 <= 0.0f) && (w_u1 <= 0.0f);
            int bfx = (w_j <= 0.0f) && (w_vj <= 0.0f);
            ute = outer_behind(s, la, lb, u0, u1, j, vj, afx, bfx, d1c);
        }
        if (ute) continue;
        v3 ne = vdiv(d1c, del);
        float pen = eth - del;
        if (bpin) {
            v3 em = vmul(vadd(vsub(p_j, p_jo), vsub(p_vj, p_vjo)), 0.5f);
            float a = 1.0f - s1, b = s1;
            float den = a * a * w_u0 + b * b * w_u1;
            if (den > EPS) {
                v3 pb = vadd(vmul(ne, pen), vmul(em, 0.5f));
                if (w_u0 > 0.0f) add_pin(s, u0, vmul(pb, fminf((a * w_u0) / den, 2.0f)));
                if (w_u1 > 0.0f) add_pin(s, u1, vmul(pb, fminf((b * w_u1) / den, 2.0f)));
            }
        } else if (apin) {
            v3 em = vmul(vadd(vsub(p_u0, p_u0o), vsub(p_u1, p_u1o)), 0.5f);
            float a = 1.0f - t1, b = t1;
            float den = a * a * w_j + b * b * w_vj;
            if (den > EPS) {
                v3 pb = vadd(vmul(vneg(ne), pen), vmul(em, 0.5f));
                if (w_j > 0.0f) add_pin(s, j, vmul(pb, fminf((a * w_j) / den, 2.0f)));
                if (w_vj > 0.0f) add_pin(s, vj, vmul(pb, fminf((b * w_vj) / den, 2.0f)));
            }
        } else {
            float we1 = (1.0f - s1) * (1.0f - s1) * w_u0 + s1 * s1 * w_u1;
            float we2 = (1.0f - t1) * (1.0f - t1) * w_j + t1 * t1 * w_vj;
            float wtot = we1 + we2;
            if (wtot > EPS) {
                v3 td = vmul(ne, pen * 0.6f);
                if (w_u0 > 0.0f) add_disp(s, u0, vmul(td, (1.0f - s1) * w_u0 / wtot));
                if (w_u1 > 0.0f) add_disp(s, u1, vmul(td, s1 * w_u1 / wtot));
                if (w_j > 0.0f) add_disp(s, j, vmul(vneg(td), (1.0f - t1) * w_j / wtot));
                if (w_vj > 0.0f) add_disp(s, vj, vmul(vneg(td), t1 * w_vj / wtot));
            }
        }
    }
}

/* dispatch_self_collision_passes, simulation/dispatch.rs:1460-1717: the
 * direct pass, or with the pair cache on the cached pass (:1556-1645) with
 * the hash and broad phase at the first substep only; the final fallback
 * runs the direct pass on the last substep. */
static void self_collision(OSim *s, int run_ee, int sub, int substeps, float dt) {
    int untangle = s->untangle_opt && s->multi_layer;
    s->rec_vt_n = s->rec_ee_n = 0;
    int force_direct = s->pair_cache && s->pair_fallback && sub + 1 == substeps;
    if (s->pair_cache && !force_direct) {
        if (untangle) k_normals(s);
        if (sub == 0) {
            build_hash(s, 0);
            memset(s->pcnt, 0, sizeof s->pcnt);
            k_pair_collect(s, dt);
        }
        k_pair_vt(s, untangle);
        if (run_ee) k_pair_ee(s, untangle);
        if (untangle) k_untangle(s);
        k_apply(s);
        return;
    }
    if (untangle) k_normals(s);
    build_hash(s, 0);
    if (run_ee && s->ne > 0) build_hash(s, 1);
    k_sc_solve(s, untangle);
    if (untangle) k_untangle(s);
    if (run_ee && s->ne > 0) k_ee(s, untangle);
    k_apply(s);
}
void ocl_set_pair_recording(OSim *s, int on) {
    s->rec = on != 0;
    s->rec_vt_n = s->rec_ee_n = 0;
}
static int cmp_rows(const uint32_t *a, const uint32_t *b, int w) {
    for (int k = 0; k < w; k++)
        if (a[k] != b[k]) return a[k] < b[k] ? -1 : 1;
    return 0;
}
static int cmp_row4(const void *a, const void *b) { return cmp_rows((const uint32_t *)a, (const uint32_t *)b, 4); }
static int cmp_row2(const void *a, const void *b) { return cmp_rows((const uint32_t *)a, (const uint32_t *)b, 2); }
static void sort3(uint32_t *r) {
    uint32_t t;
    if (r[0] > r[1]) { t = r[0]; r[0] = r[1]; r[1] = t; }
    if (r[1] > r[2]) { t = r[1]; r[1] = r[2]; r[2] = t; }
    if (r[0] > r[1]) { t = r[0]; r[0] = r[1]; r[1] = t; }
}
/* the latest pass's lists: V-T rows (vertex, a < b < c), E-E rows (e0 < e1),
 * each sorted; counts[0..1] are their lengths, rows past the capacities are
 * left out */
void ocl_get_pair_lists(OSim *s, uint32_t *vt, size_t vt_cap, uint32_t *ee, size_t ee_cap, uint32_t counts[2]) {
    for (size_t i = 0; i < s->rec_vt_n; i++) sort3(s->rec_vt + 4 * i + 1);
    for (size_t i = 0; i < s->rec_ee_n; i++) {
        uint32_t *r = s->rec_ee + 2 * i;
        if (r[0] > r[1]) { uint32_t t = r[0]; r[0] = r[1]; r[1] = t; }
    }
    if (s->rec_vt_n) qsort(s->rec_vt, s->rec_vt_n, 16, cmp_row4);
    if (s->rec_ee_n) qsort(s->rec_ee, s->rec_ee_n, 8, cmp_row2);
    counts[0] = (uint32_t)s->rec_vt_n;
    counts[1] = (uint32_t)s->rec_ee_n;
    if (vt) memcpy(vt, s->rec_vt, (s->rec_vt_n < vt_cap ? s->rec_vt_n : vt_cap) * 16);
    if (ee) memcpy(ee, s->rec_ee, (s->rec_ee_n < ee_cap ? s->rec_ee_n : ee_cap) * 8);
}
/* set_enable_pair_cache / set_enable_pair_cache_final_fallback
 * (simulation/mod.rs:805-810, :852-854) */
void ocl_set_pair_cache(OSim *s, int enable, int final_fallback) {
    s->pair_cache = enable != 0;
    s->pair_fallback = final_fallback != 0;
}
/* set_pair_cache_options, simulation/mod.rs:826-848 */
void ocl_set_pair_cache_options(OSim *s, uint32_t max_vt, uint32_t max_ee, uint32_t margin_mode, float safety,
                                float hscale, float maxh) {
    s->pair_max_vt = max_vt < 64u ? 64u : (max_vt > 262144u ? 262144u : max_vt);
    s->pair_max_ee = max_ee < 64u ? 64u : (max_ee > 262144u ? 262144u : max_ee);
    s->pair_qvt = quota_for_budget(s->pair_max_vt, (uint32_t)s->n);
    s->pair_qee = quota_for_budget(s->pair_max_ee, (uint32_t)s->n);
    s->pair_margin_mode = margin_mode == 0 ? 0 : 1;
    s->pair_safety = fminf(fmaxf(safety, 0.0f), 0.05f);
    s->pair_hscale = fminf(fmaxf(hscale, 0.0f), 4.0f);
    s->pair_maxh = fminf(fmaxf(maxh, 0.0f), 0.1f);
}
/* get_pair_cache_stats (dispatch.rs:1111-1119) and get_active_pairs
 * (dispatch.rs:1249-1290): counts = (V-T accepted, E-E accepted, stored V-T,
 * stored E-E); stored pairs in slot order, up to the capacities */
void ocl_get_active_pairs(const OSim *s, uint32_t *counts, uint32_t *vt, size_t vt_cap, uint32_t *ee, size_t ee_cap) {
    counts[0] = s->pcnt[0]; counts[1] = s->pcnt[1];
    uint32_t k = 0;
    for (size_t q = 0; q < (size_t)s->n * s->pair_qvt; q++) {
        const uint32_t *e = s->pvt + 4 * q;
        if (e[0] == 0xFFFFFFFFu) continue;
        if (vt && k < vt_cap) memcpy(vt + 4 * (size_t)k, e, 16);
        k++;
    }
    counts[2] = k;
    k = 0;
    for (size_t q = 0; q < (size_t)s->n * s->pair_qee; q++) {
        const uint32_t *e = s->pee + 4 * q;
        if (e[0] == 0xFFFFFFFFu) continue;
        if (ee && k < ee_cap) memcpy(ee + 4 * (size_t)k, e, 16);
        k++;
    }
    counts[3] = k;
}
void ocl_set_self_collision_intervals(OSim *s, int sc_interval, int ee_interval) {
    s->sc_interval = sc_interval < 1 ? 1 : sc_interval;
    s->ee_interval = ee_interval < 0 ? 0 : ee_interval;
}

/* encode_simulation_steps, simulation/dispatch.rs:7-354 (default modes:
 * coupled self-collision mode 0, no sewing priority, no edge collision) */
void ocl_step(OSim *s, float dt, int substeps) {
    if (s->n == 0) return;
    if (substeps <= 0) substeps = 20; /* base_substeps, simulation/mod.rs:673 */
    float dts = dt / (float)substeps;
    float ga = sqrtf(s->g.x * s->g.x + s->g.y * s->g.y + s->g.z * s->g.z);
    float ff = 0.5f * ga * dts * dts;
    float emd = fmaxf(s->last_eff_disp, s->last_max_disp);
    float sd = fmaxf(ff, emd / fmaxf((float)substeps, 1.0f));
    float sm = fmaxf(s->cloth_thickness * 0.8f, 0.002f);
    int risk = sd > sm * 0.25f;
    int coupled = s->coupled || (s->auto_coupled && risk);
    int hascol = s->ncols > 0 || s->ntris > 0 || s->nbones > 0;
    for (int sub = 0; sub < substeps; sub++) {
        int last = sub + 1 == substeps;
        int do_sc = s->self_collision && (s->sc_interval <= 1 || sub % s->sc_interval == 0 || last);
        int run_ee = s->ee_interval == 0 ? 0 : (s->ee_interval == 1 ? 1 : (sub % s->ee_interval == 0 || last));
        memset(s->dlam, 0, 4 * ((size_t)s->nd + 1));
        memset(s->blam, 0, 4 * ((size_t)s->nb + 1));
        memset(s->slam, 0, 4 * ((size_t)s->nsw + 1));
        k_sew_shrink(s, dts);
        k_predict(s, dts);
        for (int it = 0; it < s->iters; it++) {
            if (s->npins > 0) k_pin(s, dts);
            for (int c = 0; c < s->ndc; c++) if (s->dc_cnt[c]) k_distance(s, c, dts);
            for (int c = 0; c < s->nsc; c++) if (s->sc_cnt[c]) k_sewing(s, c, dts);
            for (int c = 0; c < s->nbc; c++) if (s->bc_cnt[c]) k_bending(s, c, dts);
            if (hascol && coupled) k_collision(s, dts);
        }
        if (hascol && !coupled) k_collision(s, dts);
        if (s->npins > 0) k_pin(s, dts);
        if (s->edge_collision && hascol && s->ne > 0) k_edge_collision(s); /* dispatch.rs:254-283 */
        if (do_sc) self_collision(s, run_ee, sub, substeps, dt);
        for (int c = 0; c < s->nsc; c++) if (s->sc_cnt[c]) k_sewing(s, c, dts); /* final sewing, dispatch.rs:323-337 */
        k_update_vel(s, dts);
    }
}

int ocl_num_vertices(const OSim *s) { return s->n; }
void ocl_set_sewing(OSim *s, float stiffness, int lock, float lock_dist, float shrink_speed) {
    s->sew_stiffness = fmaxf(stiffness, 1.0f);
    s->sew_lock = lock != 0;
    s->sew_lock_dist = fmaxf(lock_dist, 0.0f);
    s->sew_speed = fmaxf(shrink_speed, 0.0f);
}
int ocl_get_sewing(const OSim *s, int *ncolors, uint32_t *v01, float *cur, uint32_t *off, uint32_t *cnt,
                   uint32_t *rep) {
    if (ncolors) *ncolors = s->nsc;
    for (int i = 0; i < s->nsw; i++) {
        if (v01) { v01[2 * i] = s->sew[i].v0; v01[2 * i + 1] = s->sew[i].v1; }
        if (cur) cur[i] = s->sew[i].cur;
    }
    if (off) memcpy(off, s->sc_off, 4 * (size_t)s->nsc);
    if (cnt) memcpy(cnt, s->sc_cnt, 4 * (size_t)s->nsc);
    if (rep) memcpy(rep, s->rep, 4 * (size_t)s->n);
    return s->nsw;
}
void ocl_get_positions(const OSim *s, float *out) {
    for (int i = 0; i < s->n; i++) { out[3 * i] = s->x[i].x; out[3 * i + 1] = s->x[i].y; out[3 * i + 2] = s->x[i].z; }
}
void ocl_get_state(const OSim *s, float *x, float *p, float *v) {
    for (int i = 0; i < s->n; i++) {
        if (x) { x[3 * i] = s->x[i].x; x[3 * i + 1] = s->x[i].y; x[3 * i + 2] = s->x[i].z; }
        if (p) { p[3 * i] = s->p[i].x; p[3 * i + 1] = s->p[i].y; p[3 * i + 2] = s->p[i].z; }
        if (v) { v[3 * i] = s->v[i].x; v[3 * i + 1] = s->v[i].y; v[3 * i + 2] = s->v[i].z; }
    }
}
/* set_positions_and_velocities, simulation/dispatch.rs:953-988 */
void ocl_set_state(OSim *s, const float *x, const float *v) {
    for (int i = 0; i < s->n; i++) {
        s->x[i] = V3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
        s->p[i] = s->x[i];
        s->v[i] = v ? V3(v[3 * i], v[3 * i + 1], v[3 * i + 2]) : V3(0, 0, 0);
    }
}
void ocl_counts(const OSim *s, int *o) {
    o[0] = s->nd; o[1] = s->nb; o[2] = s->ndc; o[3] = s->nbc; o[4] = s->ne; o[5] = (int)s->table;
    o[6] = s->num_virtual; o[7] = s->multi_layer;
}
void ocl_get_distance(const OSim *s, uint32_t *v01, float *rest, float *tc, float *cc, uint32_t *type) {
    for (int i = 0; i < s->nd; i++) {
        v01[2 * i] = s->dist[i].v0; v01[2 * i + 1] = s->dist[i].v1;
        rest[i] = s->dist[i].rest; tc[i] = s->dist[i].tc; cc[i] = s->dist[i].cc; type[i] = s->dist[i].type;
    }
}
void ocl_get_bending(const OSim *s, uint32_t *v, float *rest, float *comp, float *pad0) {
    for (int i = 0; i < s->nb; i++) {
        v[4 * i] = s->bend[i].v0; v[4 * i + 1] = s->bend[i].v1; v[4 * i + 2] = s->bend[i].v2; v[4 * i + 3] = s->bend[i].v3;
        rest[i] = s->bend[i].rest; comp[i] = s->bend[i].comp; pad0[i] = s->bend[i].pad0;
    }
}
void ocl_get_bending_gate(const OSim *s, float *pad1) {
    for (int i = 0; i < s->nb; i++) pad1[i] = s->bend[i].pad1;
}
void ocl_get_dist_colors(const OSim *s, uint32_t *off, uint32_t *cnt) {
    memcpy(off, s->dc_off, 4 * (size_t)s->ndc); memcpy(cnt, s->dc_cnt, 4 * (size_t)s->ndc);
}
void ocl_get_bend_colors(const OSim *s, uint32_t *off, uint32_t *cnt) {
    memcpy(off, s->bc_off, 4 * (size_t)s->nbc); memcpy(cnt, s->bc_cnt, 4 * (size_t)s->nbc);
}
void ocl_get_edges(const OSim *s, uint32_t *e2, uint32_t *bits) {
    memcpy(e2, s->edges, 8 * (size_t)s->ne);
    memcpy(bits, s->ebits, 4 * (size_t)((s->ne + 31) / 32));
}
int ocl_topology_sizes(const OSim *s, int *adj_n, int *th_n, int *star_n) {
    *adj_n = (int)s->adj_off[s->n]; *th_n = (int)s->th_off[s->n]; *star_n = (int)s->star_off[s->n];
    return s->n;
}
void ocl_get_topology(const OSim *s, uint32_t *adj_off, uint32_t *adj_idx, uint32_t *th_off, uint32_t *th_idx,
                      float *th_rest, float *local_len, uint32_t *star_off, uint32_t *star_idx, uint32_t *island,
                      uint32_t *layer) {
    int n = s->n;
    memcpy(adj_off, s->adj_off, 4 * ((size_t)n + 1)); memcpy(adj_idx, s->adj_idx, 4 * (size_t)s->adj_off[n]);
    memcpy(th_off, s->th_off, 4 * ((size_t)n + 1)); memcpy(th_idx, s->th_idx, 4 * (size_t)s->th_off[n]);
    memcpy(th_rest, s->th_rest, 4 * (size_t)s->th_off[n]); memcpy(local_len, s->local_len, 4 * (size_t)n);
    memcpy(star_off, s->star_off, 4 * ((size_t)n + 1)); memcpy(star_idx, s->star_idx, 8 * (size_t)s->star_off[n]);
    memcpy(island, s->island, 4 * (size_t)n); memcpy(layer, s->layer, 4 * (size_t)n);
}
float ocl_cell_size(const OSim *s) { return s->cell; }
void ocl_build_hash(OSim *s, int which, uint32_t *cs, uint32_t *srt) {
    build_hash(s, which);
    memcpy(cs, which == 0 ? s->cs : s->ecs, 4 * ((size_t)s->table + 1));
    memcpy(srt, which == 0 ? s->srt : s->esrt, 4 * (size_t)(which == 0 ? s->n : s->ne));
}
void ocl_get_mesh_triangles(const OSim *s, float *o) {
    for (int t = 0; t < s->ntris; t++) {
        const OTri *q = &s->tris[t];
        float r[16] = {q->p0.x, q->p0.y, q->p0.z, q->fric, q->p1.x, q->p1.y, q->p1.z, q->thick,
                       q->p2.x, q->p2.y, q->p2.z, q->rest, 0, 0, 0, 0};
        memcpy(&r[12], &q->flags, 4);
        memcpy(o + 16 * t, r, sizeof r);
    }
}
