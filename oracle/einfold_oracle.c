/*
 * ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the inner loops of einfold's kernel layer
 * (crates/einfold-kernels), used only by tests/, by __graft_entry__.smoke() to
 * check its result, and by bench.py's CPU-baseline leg. Nothing in the product path
 * (einfold_b200/, include/) links or calls this file.
 *
 * Each function names the reference lines it follows. Floating-point sums are
 * done in the reference's order with separate multiply and add (built with
 * -ffp-contract=off), as Rust never fuses them, so the dense and
 * discrimination results are the reference's bits. The fused tile's block
 * products follow a fixed k order without fusing; the reference calls the
 * matrixmultiply crate there, whose bits depend on the CPU, so that part is
 * pinned by tolerance only.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* SplitMix64 (crates/einfold-testkit/src/rng.rs:17-28)                     */
/* ------------------------------------------------------------------------ */

uint64_t ef_rng_seeded(uint64_t seed, uint64_t salt) {
    return (seed * 0x2545f4914f6cdd1dULL) ^ salt;
}

uint64_t ef_rng_next(uint64_t *state) {
    uint64_t z;
    *state += 0x9e3779b97f4a7c15ULL;
    z = *state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

/* Fills out[n] with next_u64 draws. */
void ef_rng_fill(uint64_t *state, uint64_t *out, int64_t n) {
    for (int64_t i = 0; i < n; i++) out[i] = ef_rng_next(state);
}

/* Fills out[n] with unit() draws: 53 random bits in [0, 1) (rng.rs:41-43). */
void ef_rng_units(uint64_t *state, double *out, int64_t n) {
    for (int64_t i = 0; i < n; i++)
        out[i] = (double)(ef_rng_next(state) >> 11) / (double)(1ULL << 53);
}

/* ------------------------------------------------------------------------ */
/* par_tasks (dense.rs:142-168): task i runs on thread i % threads.          */
/* ------------------------------------------------------------------------ */

typedef void (*ef_task_fn)(void *ctx, int64_t task);

typedef struct {
    ef_task_fn fn;
    void *ctx;
    int64_t tasks;
    int threads;
    int tid;
} ef_worker;

static void *ef_worker_main(void *p) {
    ef_worker *w = (ef_worker *)p;
    for (int64_t t = w->tid; t < w->tasks; t += w->threads) w->fn(w->ctx, t);
    return NULL;
}

static void ef_par_tasks(int64_t tasks, int threads, ef_task_fn fn, void *ctx) {
    if (threads < 1) threads = 1;
    if (tasks < 1) return;
    if (threads > tasks) threads = (int)tasks;
    if (threads == 1) {
        for (int64_t t = 0; t < tasks; t++) fn(ctx, t);
        return;
    }
    pthread_t th[256];
    ef_worker w[256];
    if (threads > 256) threads = 256;
    for (int i = 0; i < threads; i++) {
        w[i].fn = fn; w[i].ctx = ctx; w[i].tasks = tasks; w[i].threads = threads; w[i].tid = i;
        pthread_create(&th[i], NULL, ef_worker_main, &w[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
}

/* ------------------------------------------------------------------------ */
/* Dense accumulate (dense.rs:706-770)                                      */
/* ------------------------------------------------------------------------ */

#define EF_XB 256
#define EF_YB 2048
#define EF_ZB 4096
#define EF_FEW_CELLS 4096
#define EF_VALUED 2

typedef struct {
    const double *a; const uint8_t *held; const double *b;
    int64_t nx, nz, ny, per_batch;
    double *out;
    double **parts;
    int64_t column_blocks;
} ef_acc_ctx;

static inline void ef_acc_add(const ef_acc_ctx *c, double *row, int64_t width, int64_t x, int64_t z, int64_t y0) {
    if (c->held[x * c->nz + z] == EF_VALUED) {
        double v = c->a[x * c->nz + z];
        int64_t start = ((x / c->per_batch) * c->nz + z) * c->ny + y0;
        const double *brow = c->b + start;
        for (int64_t y = 0; y < width; y++) {
            double p = v * brow[y];
            row[y] = row[y] + p;
        }
    }
}

static void ef_acc_block(void *p, int64_t t) {
    ef_acc_ctx *c = (ef_acc_ctx *)p;
    int64_t x0 = (t / c->column_blocks) * EF_XB, y0 = (t % c->column_blocks) * EF_YB;
    int64_t x1 = x0 + EF_XB < c->nx ? x0 + EF_XB : c->nx;
    int64_t width = c->ny - y0 < EF_YB ? c->ny - y0 : EF_YB;
    for (int64_t x = x0; x < x1; x++) {
        double *row = c->out + x * c->ny + y0;
        for (int64_t y = 0; y < width; y++) row[y] = 0.0;
        for (int64_t z = 0; z < c->nz; z++) ef_acc_add(c, row, width, x, z, y0);
    }
}

static void ef_acc_zpart(void *p, int64_t t) {
    ef_acc_ctx *c = (ef_acc_ctx *)p;
    double *part = c->parts[t];
    int64_t z1 = (t + 1) * EF_ZB < c->nz ? (t + 1) * EF_ZB : c->nz;
    for (int64_t i = 0; i < c->nx * c->ny; i++) part[i] = 0.0;
    for (int64_t z = t * EF_ZB; z < z1; z++)
        for (int64_t x = 0; x < c->nx; x++) ef_acc_add(c, part + x * c->ny, c->ny, x, z, 0);
}

/* out[nx*ny] = accumulate(a[nx*nz], held[nx*nz], b[nw*nz*ny]); returns 0. */
int ef_dense_accumulate(const double *a, const uint8_t *held, const double *b, int64_t nx, int64_t nz,
                        int64_t ny, int64_t per_batch, double *out, int threads) {
    ef_acc_ctx c = {a, held, b, nx, nz, ny, per_batch > 0 ? per_batch : 1, out, NULL, 0};
    if (nx * ny >= EF_FEW_CELLS) {
        int64_t row_blocks = (nx + EF_XB - 1) / EF_XB;
        c.column_blocks = (ny + EF_YB - 1) / EF_YB;
        ef_par_tasks(row_blocks * c.column_blocks, threads, ef_acc_block, &c);
    } else {
        int64_t tasks = (nz + EF_ZB - 1) / EF_ZB;
        c.parts = (double **)calloc((size_t)(tasks > 0 ? tasks : 1), sizeof(double *));
        for (int64_t t = 0; t < tasks; t++) c.parts[t] = (double *)malloc(sizeof(double) * (size_t)(nx * ny > 0 ? nx * ny : 1));
        ef_par_tasks(tasks, threads, ef_acc_zpart, &c);
        for (int64_t i = 0; i < nx * ny; i++) out[i] = 0.0;
        for (int64_t t = 0; t < tasks; t++) {
            for (int64_t i = 0; i < nx * ny; i++) out[i] = out[i] + c.parts[t][i];
            free(c.parts[t]);
        }
        free(c.parts);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* LSD radix ranks (discriminate.rs:103-156 radix, :280-292 ranks_of_words)  */
/* ------------------------------------------------------------------------ */

#define EF_CHUNK 65536

typedef struct { uint64_t w; uint32_t r; } ef_pair;

typedef struct {
    ef_pair *pairs, *next;
    int64_t n; int chunks; int shift;
    int64_t *bounds;       /* chunks + 1 */
    int64_t (*counts)[256];/* per chunk */
    int64_t (*at)[256];    /* per chunk: where each byte's region starts */
} ef_radix_ctx;

static void ef_radix_count(void *p, int64_t c) {
    ef_radix_ctx *x = (ef_radix_ctx *)p;
    int64_t *cnt = x->counts[c];
    memset(cnt, 0, sizeof(int64_t) * 256);
    for (int64_t i = x->bounds[c]; i < x->bounds[c + 1]; i++) cnt[(x->pairs[i].w >> x->shift) & 0xff]++;
}

static void ef_radix_scatter(void *p, int64_t c) {
    ef_radix_ctx *x = (ef_radix_ctx *)p;
    int64_t *at = x->at[c];
    for (int64_t i = x->bounds[c]; i < x->bounds[c + 1]; i++) {
        int b = (int)((x->pairs[i].w >> x->shift) & 0xff);
        x->next[at[b]++] = x->pairs[i];
    }
}

/* Sorts (word, row) pairs by word, stably; writes the sorted rows to order[n]
 * and words to sorted[n] (either may be NULL). */
void ef_radix_sort_words(const uint64_t *words, int64_t n, int threads, uint32_t *order, uint64_t *sorted) {
    if (n <= 0) return;
    int64_t want = (n + EF_CHUNK - 1) / EF_CHUNK;
    int chunks = threads < want ? threads : (int)want;
    if (chunks < 1) chunks = 1;
    ef_radix_ctx x;
    x.n = n; x.chunks = chunks;
    x.pairs = (ef_pair *)malloc(sizeof(ef_pair) * (size_t)n);
    x.next = (ef_pair *)malloc(sizeof(ef_pair) * (size_t)n);
    x.bounds = (int64_t *)malloc(sizeof(int64_t) * (size_t)(chunks + 1));
    x.counts = (int64_t (*)[256])malloc(sizeof(int64_t) * 256 * (size_t)chunks);
    x.at = (int64_t (*)[256])malloc(sizeof(int64_t) * 256 * (size_t)chunks);
    for (int c = 0; c <= chunks; c++) x.bounds[c] = n * c / chunks;
    uint64_t any = 0, all = ~0ULL;
    for (int64_t i = 0; i < n; i++) {
        x.pairs[i].w = words[i]; x.pairs[i].r = (uint32_t)i;
        any |= words[i]; all &= words[i];
    }
    for (int shift = 0; shift < 64; shift += 8) {
        if ((((any ^ all) >> shift) & 0xff) == 0) continue;
        x.shift = shift;
        ef_par_tasks(chunks, threads, ef_radix_count, &x);
        /* Regions byte-major, then chunk (discriminate.rs:127-139). */
        int64_t pos = 0;
        for (int b = 0; b < 256; b++)
            for (int c = 0; c < chunks; c++) { x.at[c][b] = pos; pos += x.counts[c][b]; }
        ef_par_tasks(chunks, threads, ef_radix_scatter, &x);
        ef_pair *t = x.pairs; x.pairs = x.next; x.next = t;
    }
    for (int64_t i = 0; i < n; i++) {
        if (order) order[i] = x.pairs[i].r;
        if (sorted) sorted[i] = x.pairs[i].w;
    }
    free(x.pairs); free(x.next); free(x.bounds); free(x.counts); free(x.at);
}

/* rank[n] and first[] of words in their order; returns the number of ranks. */
int64_t ef_ranks_of_words(const uint64_t *words, int64_t n, int threads, uint32_t *rank, uint32_t *first) {
    if (n <= 0) return 0;
    uint32_t *order = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    uint64_t *sorted = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    ef_radix_sort_words(words, n, threads, order, sorted);
    int64_t k = 0;
    for (int64_t i = 0; i < n; i++) {
        if (i == 0 || sorted[i] != sorted[i - 1]) first[k++] = order[i];
        rank[order[i]] = (uint32_t)(k - 1);
    }
    free(order); free(sorted);
    return k;
}

/* ------------------------------------------------------------------------ */
/* MSD byte sort (discriminate.rs:165-209 by_bytes) and ranks (:212-235)     */
/* ------------------------------------------------------------------------ */

#define EF_SMALL 16

typedef struct { const uint8_t *data; const int64_t *off; } ef_keys;

static inline int ef_key_len(const ef_keys *k, uint32_t i) { return (int)(k->off[i + 1] - k->off[i]); }

/* Rust slice order from `depth` on: bytewise, a key that ends first sorts first. */
static int ef_rest_cmp(const ef_keys *k, uint32_t a, uint32_t b, int64_t depth) {
    int64_t la = k->off[a + 1] - k->off[a] - depth, lb = k->off[b + 1] - k->off[b] - depth;
    if (la < 0) la = 0;
    if (lb < 0) lb = 0;
    int64_t m = la < lb ? la : lb;
    int c = m > 0 ? memcmp(k->data + k->off[a] + depth, k->data + k->off[b] + depth, (size_t)m) : 0;
    if (c) return c;
    return (la > lb) - (la < lb);
}

static inline int ef_bucket(const ef_keys *k, uint32_t i, int64_t depth) {
    return depth < k->off[i + 1] - k->off[i] ? (int)k->data[k->off[i] + depth] + 1 : 0;
}

void ef_by_bytes(const uint8_t *data, const int64_t *off, uint32_t *index, int64_t n) {
    ef_keys k = {data, off};
    typedef struct { int64_t lo, hi, depth; } item;
    int64_t cap = 1024, top = 0;
    item *work = (item *)malloc(sizeof(item) * (size_t)cap);
    uint32_t *scratch = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    work[top++] = (item){0, n, 0};
    while (top > 0) {
        item it = work[--top];
        uint32_t *ix = index + it.lo;
        int64_t len = it.hi - it.lo;
        if (len <= EF_SMALL) {
            /* Stable insertion sort by the rest of each key. */
            for (int64_t i = 1; i < len; i++) {
                uint32_t v = ix[i];
                int64_t j = i;
                while (j > 0 && ef_rest_cmp(&k, ix[j - 1], v, it.depth) > 0) { ix[j] = ix[j - 1]; j--; }
                ix[j] = v;
            }
            continue;
        }
        int64_t start[259];
        memset(start, 0, sizeof(start));
        for (int64_t i = 0; i < len; i++) start[ef_bucket(&k, ix[i], it.depth) + 1]++;
        int nonzero = 0;
        for (int b = 0; b < 259; b++) nonzero += start[b] > 0;
        if (start[1] == 0 && nonzero == 1) {
            if (top == cap) { cap *= 2; work = (item *)realloc(work, sizeof(item) * (size_t)cap); }
            work[top++] = (item){it.lo, it.hi, it.depth + 1};
            continue;
        }
        for (int b = 1; b < 258; b++) start[b] += start[b - 1];
        int64_t at[258];
        memcpy(at, start, sizeof(at));
        for (int64_t i = 0; i < len; i++) {
            int b = ef_bucket(&k, ix[i], it.depth);
            scratch[at[b]++] = ix[i];
        }
        memcpy(ix, scratch, sizeof(uint32_t) * (size_t)len);
        for (int b = 1; b < 257; b++) {
            if (start[b + 1] - start[b] > 1) {
                if (top == cap) { cap *= 2; work = (item *)realloc(work, sizeof(item) * (size_t)cap); }
                work[top++] = (item){it.lo + start[b], it.lo + start[b + 1], it.depth + 1};
            }
        }
    }
    free(work); free(scratch);
}

/* Ranks of byte keys (ranks(), discriminate.rs:212-235, by_bytes branch). */
int64_t ef_ranks_of_bytes(const uint8_t *data, const int64_t *off, int64_t n, uint32_t *rank, uint32_t *first) {
    if (n <= 0) return 0;
    uint32_t *index = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
    for (int64_t i = 0; i < n; i++) index[i] = (uint32_t)i;
    ef_by_bytes(data, off, index, n);
    ef_keys k = {data, off};
    int64_t count = 0;
    int64_t prev = -1;
    for (int64_t i = 0; i < n; i++) {
        uint32_t r = index[i];
        int same = prev >= 0 && ef_key_len(&k, r) == ef_key_len(&k, (uint32_t)prev) &&
                   memcmp(data + off[r], data + off[prev], (size_t)ef_key_len(&k, r)) == 0;
        if (!same) { first[count++] = r; prev = r; }
        rank[r] = (uint32_t)(count - 1);
    }
    free(index);
    return count;
}

/* ------------------------------------------------------------------------ */
/* Gustavson's product over blocks of 256 x ranks (discriminate.rs:548-584)  */
/* ------------------------------------------------------------------------ */

typedef struct {
    /* a's joining rows in (x, z) order, with ties broken by factor bits */
    const uint32_t *a_rows; const int64_t *a_start; const uint32_t *a_z;
    const double *a_f; const uint8_t *a_valid;
    /* b laid out by z: y rank and factor per entry */
    const int64_t *b_start; const uint32_t *b_y; const double *b_f; const uint8_t *b_valid;
    int64_t nx, ny;
    /* per block output */
    int64_t *counts; uint32_t **gx; uint32_t **gy; double **gs; uint8_t **gv;
} ef_gus_ctx;

static int ef_cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

static void ef_gus_block(void *p, int64_t t) {
    ef_gus_ctx *c = (ef_gus_ctx *)p;
    double *acc = (double *)calloc((size_t)c->ny, sizeof(double));
    uint8_t *valued = (uint8_t *)calloc((size_t)c->ny, 1);
    uint8_t *reached = (uint8_t *)calloc((size_t)c->ny, 1);
    uint32_t *touched = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)c->ny);
    int64_t cap = 1024, n = 0;
    uint32_t *gx = (uint32_t *)malloc(sizeof(uint32_t) * cap), *gy = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    double *gs = (double *)malloc(sizeof(double) * cap);
    uint8_t *gv = (uint8_t *)malloc((size_t)cap);
    int64_t x1 = (t + 1) * EF_XB < c->nx ? (t + 1) * EF_XB : c->nx;
    for (int64_t xr = t * EF_XB; xr < x1; xr++) {
        int64_t nt = 0;
        for (int64_t i = c->a_start[xr]; i < c->a_start[xr + 1]; i++) {
            uint32_t r = c->a_rows[i];
            uint32_t zr = c->a_z[r];
            int av = c->a_valid[r];
            double p = c->a_f[r];
            for (int64_t j = c->b_start[zr]; j < c->b_start[zr + 1]; j++) {
                uint32_t yr = c->b_y[j];
                if (!reached[yr]) { reached[yr] = 1; touched[nt++] = yr; }
                if (av && c->b_valid[j]) {
                    double q = c->b_f[j];
                    double pq = p * q;
                    acc[yr] = acc[yr] + pq;
                    valued[yr] = 1;
                }
            }
        }
        qsort(touched, (size_t)nt, sizeof(uint32_t), ef_cmp_u32);
        for (int64_t i = 0; i < nt; i++) {
            uint32_t yr = touched[i];
            if (n == cap) {
                cap *= 2;
                gx = (uint32_t *)realloc(gx, sizeof(uint32_t) * cap);
                gy = (uint32_t *)realloc(gy, sizeof(uint32_t) * cap);
                gs = (double *)realloc(gs, sizeof(double) * cap);
                gv = (uint8_t *)realloc(gv, (size_t)cap);
            }
            gx[n] = (uint32_t)xr; gy[n] = yr; gs[n] = acc[yr]; gv[n] = valued[yr]; n++;
            acc[yr] = 0.0; valued[yr] = 0; reached[yr] = 0;
        }
    }
    free(acc); free(valued); free(reached); free(touched);
    c->counts[t] = n; c->gx[t] = gx; c->gy[t] = gy; c->gs[t] = gs; c->gv[t] = gv;
}

/* Runs the product; returns the number of groups, written to the out arrays
 * (capacity cap), or -(needed) when cap is too small. */
int64_t ef_gustavson(const uint32_t *a_rows, const int64_t *a_start, const uint32_t *a_z, const double *a_f,
                     const uint8_t *a_valid, const int64_t *b_start, const uint32_t *b_y, const double *b_f,
                     const uint8_t *b_valid, int64_t nx, int64_t ny, int threads, int64_t cap,
                     uint32_t *out_x, uint32_t *out_y, double *out_sum, uint8_t *out_valued) {
    int64_t blocks = (nx + EF_XB - 1) / EF_XB;
    ef_gus_ctx c = {a_rows, a_start, a_z, a_f, a_valid, b_start, b_y, b_f, b_valid, nx, ny ? ny : 1,
                    NULL, NULL, NULL, NULL, NULL};
    c.counts = (int64_t *)calloc((size_t)(blocks + 1), sizeof(int64_t));
    c.gx = (uint32_t **)calloc((size_t)(blocks + 1), sizeof(void *));
    c.gy = (uint32_t **)calloc((size_t)(blocks + 1), sizeof(void *));
    c.gs = (double **)calloc((size_t)(blocks + 1), sizeof(void *));
    c.gv = (uint8_t **)calloc((size_t)(blocks + 1), sizeof(void *));
    ef_par_tasks(blocks, threads, ef_gus_block, &c);
    int64_t total = 0;
    for (int64_t t = 0; t < blocks; t++) total += c.counts[t];
    int64_t pos = 0;
    if (total <= cap) {
        for (int64_t t = 0; t < blocks; t++) {
            memcpy(out_x + pos, c.gx[t], sizeof(uint32_t) * (size_t)c.counts[t]);
            memcpy(out_y + pos, c.gy[t], sizeof(uint32_t) * (size_t)c.counts[t]);
            memcpy(out_sum + pos, c.gs[t], sizeof(double) * (size_t)c.counts[t]);
            memcpy(out_valued + pos, c.gv[t], (size_t)c.counts[t]);
            pos += c.counts[t];
        }
    }
    for (int64_t t = 0; t < blocks; t++) { free(c.gx[t]); free(c.gy[t]); free(c.gs[t]); free(c.gv[t]); }
    free(c.counts); free(c.gx); free(c.gy); free(c.gs); free(c.gv);
    return total <= cap ? total : -total;
}

/* ------------------------------------------------------------------------ */
/* Expressions (crates/einfold-ir/src/expression.rs:72-114, 168-178)         */
/* ------------------------------------------------------------------------ */

typedef struct { int32_t kind, op, col, pad; double lit; } ef_node; /* postfix; kind 0 col,1 lit,2 un,3 bin */

static inline double ef_unary(int op, double x) {
    switch (op) {
        case 0: return -x;
        case 1: return fabs(x);
        case 2: return exp(x);
        default: return log(x);
    }
}

static inline double ef_binary(int op, double a, double b) {
    switch (op) {
        case 0: return a + b;
        case 1: return a - b;
        case 2: return a * b;
        case 3: return a / b;
        default: return pow(a, b);
    }
}

/* Evaluates a postfix expression whose column nodes read vals[operand] (the
 * "column" field picks one of the values given per operand slot: the caller
 * resolves (operand, column) to slot = col). */
static double ef_eval(const ef_node *nodes, int n, const double *slots) {
    double st[64];
    int sp = 0;
    for (int i = 0; i < n; i++) {
        const ef_node *e = &nodes[i];
        if (e->kind == 0) st[sp++] = slots[e->col];
        else if (e->kind == 1) st[sp++] = e->lit;
        else if (e->kind == 2) st[sp - 1] = ef_unary(e->op, st[sp - 1]);
        else { double b = st[--sp]; st[sp - 1] = ef_binary(e->op, st[sp - 1], b); }
    }
    return st[0];
}

/* Evaluates expr over n rows, slot s of row r at slots[s * n + r]. */
void ef_eval_rows(const ef_node *nodes, int n_nodes, const double *slots, int n_slots, int64_t n, double *out) {
    double v[32];
    for (int64_t r = 0; r < n; r++) {
        for (int s = 0; s < n_slots; s++) v[s] = slots[s * n + r];
        out[r] = ef_eval(nodes, n_nodes, v);
    }
}

/* ------------------------------------------------------------------------ */
/* The fused tile (fused.rs:694-1019), with overflows (:1024-1028) and       */
/* Bounds::hold (:1058-1086).                                                */
/* ------------------------------------------------------------------------ */

#define EF_XT 64
#define EF_JT 64

typedef struct {
    /* shape */
    int64_t nx, ne, nj, ny;
    int64_t local_nx, local_nj;
    /* weight: 0 = exp softmax, 1 = expression of the score */
    int weight_kind;
    int scale_kind; double scale_c; /* 0 one, 1 times, 2 over */
    int shifted;
    int normalizer; /* 0 kept, 1 joined, 2 none */
    const ef_node *weight_nodes; int weight_n;
    /* scores: 0 = product q[x][e]·kt[e][j]; 1 = expression */
    int scores_kind;
    const double *q; const double *kt;
    const ef_node *score_nodes; int score_n;
    /* expression columns: slot s reads matrix mats[s], operand side[s] (0 q: [x][e], 1 k: [e][j]) */
    int n_slots; const double *const *mats; const int *side;
    /* mask: conditions as (comparison, offset) of x against j */
    int n_mask; const int *mask_cmp; const int64_t *mask_off;
    /* values */
    const double *v; const uint8_t *finite; const double *largest; const double *smallest;
    /* outputs */
    double *out;        /* [nx][ny] */
    int64_t *visited;   /* per tile */
    uint8_t *overflowed;/* per tile */
} ef_fused_ctx;

static inline double ef_scale(const ef_fused_ctx *c, double p) {
    if (c->scale_kind == 0) return p;
    if (c->scale_kind == 1) return p * c->scale_c;
    return p / c->scale_c;
}

/* allowed(x) (fused.rs:350-368). */
static void ef_allowed(const ef_fused_ctx *c, int64_t x, int64_t *lo_out, int64_t *hi_out) {
    int64_t group_start = (x / c->local_nx) * c->local_nj;
    __int128 xx = x % c->local_nx;
    __int128 n = c->local_nj;
    __int128 lo = 0, hi = n;
    for (int i = 0; i < c->n_mask; i++) {
        __int128 bound = xx - (__int128)c->mask_off[i];
        switch (c->mask_cmp[i]) {
            case 3: if (bound + 1 < hi) hi = bound + 1; break;  /* >= */
            case 2: if (bound < hi) hi = bound; break;          /* >  */
            case 1: if (bound > lo) lo = bound; break;          /* <= */
            default: if (bound + 1 > lo) lo = bound + 1; break; /* <  */
        }
    }
    __int128 l = lo < 0 ? 0 : (lo > n ? n : lo);
    __int128 h = hi > lo ? hi : lo;
    h = h < 0 ? 0 : (h > n ? n : h);
    *lo_out = group_start + (int64_t)l;
    *hi_out = group_start + (int64_t)h;
}

void ef_fused_allowed(const int64_t *shape, int n_mask, const int *cmp, const int64_t *off, int64_t x,
                      int64_t *lo, int64_t *hi) {
    ef_fused_ctx c;
    memset(&c, 0, sizeof(c));
    c.local_nx = shape[0]; c.local_nj = shape[1];
    c.n_mask = n_mask; c.mask_cmp = cmp; c.mask_off = off;
    ef_allowed(&c, x, lo, hi);
}

static int ef_overflows(double z, const double *a, int special_weight, const uint8_t *special_value, int64_t ny) {
    if (special_weight) return 0;
    if (!isfinite(z)) return 1;
    for (int64_t y = 0; y < ny; y++)
        if (!special_value[y] && !isfinite(a[y])) return 1;
    return 0;
}

/* Bounds::hold; z_present says whether there is a normalizer. */
int ef_bounds_hold(double heaviest, double lightest, double largest, double smallest, int64_t terms_n,
                   int z_present, double z, const double *results, const uint8_t *special, int64_t n) {
    double terms = 2.0 * (double)terms_n;
    int finite = isfinite(heaviest * largest * terms);
    if (finite && z_present) {
        double quotient = heaviest / fabs(z);
        finite = isfinite(quotient) && isfinite(quotient * largest * terms);
    }
    double inverse = z_present ? 1.0 / fabs(z) : 1.0;
    double tiniest = 4.9406564584124654e-324; /* 2^-1074 */
    double lost = terms * tiniest * (inverse + largest + 1.0);
    double rounding = 2.220446049250313e-16 / 4.0;
    double normal = 2.0 * 2.2250738585072014e-308;
    int no_underflow = smallest == INFINITY;
    if (!no_underflow) {
        no_underflow = lightest * smallest >= normal;
        if (no_underflow && z_present) {
            double quotient = lightest / fabs(z);
            no_underflow = quotient >= normal && quotient * smallest >= normal;
        }
    }
    if (!finite) return 0;
    if (no_underflow) return 1;
    for (int64_t i = 0; i < n; i++)
        if (!special[i] && !(lost <= rounding * fabs(results[i]))) return 0;
    return 1;
}

static void ef_fused_tile(void *p, int64_t t) {
    ef_fused_ctx *c = (ef_fused_ctx *)p;
    int64_t nx = c->nx, ne = c->ne, nj = c->nj, ny = c->ny;
    int64_t x0 = t * EF_XT, x1 = (t + 1) * EF_XT < nx ? (t + 1) * EF_XT : nx;
    int64_t rows = x1 - x0;
    int map = c->weight_kind == 1;
    int shifted = map ? 0 : c->shifted;
    int unnormalized = c->normalizer == 2;
    double *m = (double *)malloc(sizeof(double) * rows);
    double *z = (double *)calloc((size_t)rows, sizeof(double));
    double *a = c->out + x0 * ny;
    double *block = (double *)malloc(sizeof(double) * EF_XT * EF_JT);
    uint8_t *special_weight = (uint8_t *)calloc((size_t)rows, 1);
    uint8_t *special_value = (uint8_t *)calloc((size_t)(rows * ny), 1);
    double *high = (double *)malloc(sizeof(double) * rows);
    double *light = (double *)malloc(sizeof(double) * rows);
    int64_t *terms = (int64_t *)calloc((size_t)rows, sizeof(int64_t));
    double *row_largest = (double *)calloc((size_t)rows, sizeof(double));
    double *row_smallest = (double *)malloc(sizeof(double) * rows);
    double *low = (double *)malloc(sizeof(double) * rows);
    int64_t *slo = (int64_t *)malloc(sizeof(int64_t) * rows), *shi = (int64_t *)malloc(sizeof(int64_t) * rows);
    int64_t visited = 0;
    int overflowed = 0;
    for (int64_t r = 0; r < rows; r++) {
        m[r] = shifted ? -INFINITY : 0.0;
        high[r] = -INFINITY; light[r] = INFINITY; row_smallest[r] = INFINITY; low[r] = INFINITY;
        for (int64_t y = 0; y < ny; y++) a[r * ny + y] = 0.0;
    }
    int64_t first = nj, last = 0;
    for (int64_t x = x0; x < x1; x++) {
        int64_t lo, hi;
        ef_allowed(c, x, &lo, &hi);
        if (lo < hi) { if (lo < first) first = lo; if (hi > last) last = hi; }
    }
    double slots[32];
    for (int64_t j0 = first - first % EF_JT; j0 < last; j0 += EF_JT) {
        int64_t width = EF_JT < nj - j0 ? EF_JT : nj - j0;
        int any = 0, full = 1;
        for (int64_t r = 0; r < rows; r++) {
            int64_t lo, hi;
            ef_allowed(c, x0 + r, &lo, &hi);
            lo = lo < j0 ? j0 : (lo > j0 + width ? j0 + width : lo);
            hi = hi < j0 ? j0 : (hi > j0 + width ? j0 + width : hi);
            slo[r] = lo - j0; shi[r] = hi - j0;
            if (slo[r] < shi[r]) any = 1;
            if (!(slo[r] == 0 && shi[r] == width)) full = 0;
        }
        if (!any) continue;
        visited++;
        (void)full;
        if (c->scores_kind == 0) {
            for (int64_t r = 0; r < rows; r++)
                for (int64_t j = 0; j < width; j++) {
                    double s = 0.0;
                    for (int64_t e = 0; e < ne; e++) {
                        double pr = c->q[(x0 + r) * ne + e] * c->kt[e * nj + j0 + j];
                        s = s + pr;
                    }
                    block[r * width + j] = s;
                }
        } else {
            for (int64_t r = 0; r < rows; r++)
                for (int64_t j = 0; j < width; j++) {
                    double s = 0.0;
                    for (int64_t e = 0; e < ne; e++) {
                        for (int sl = 0; sl < c->n_slots; sl++)
                            slots[sl] = c->side[sl] == 0 ? c->mats[sl][(x0 + r) * ne + e]
                                                         : c->mats[sl][e * nj + j0 + j];
                        double val = ef_eval(c->score_nodes, c->score_n, slots);
                        s = e == 0 ? val : s + val;
                    }
                    block[r * width + j] = s;
                }
        }
        for (int64_t r = 0; r < rows; r++) {
            int64_t lo = slo[r], hi = shi[r];
            if (lo >= hi) continue;
            terms[r] += hi - lo;
            for (int64_t j = j0 + lo; j < j0 + hi; j++) {
                if (c->largest[j] > row_largest[r]) row_largest[r] = c->largest[j];
                if (c->smallest[j] < row_smallest[r]) row_smallest[r] = c->smallest[j];
            }
            double *sc = block + r * width + lo;
            int64_t cnt = hi - lo;
            if (map) {
                for (int64_t i = 0; i < cnt; i++) { slots[0] = sc[i]; sc[i] = ef_eval(c->weight_nodes, c->weight_n, slots); }
                for (int64_t i = 0; i < cnt; i++) if (!isfinite(sc[i])) overflowed = 1;
                for (int64_t j = lo; j < hi; j++) if (!c->finite[j0 + j]) overflowed = 1;
                for (int64_t i = 0; i < cnt; i++) {
                    double w = fabs(sc[i]);
                    high[r] = fmax(high[r], w); /* f64::max ignores NaN */
                    if (w != 0.0 && w < light[r]) light[r] = w;
                }
                double sum = 0.0;
                for (int64_t i = 0; i < cnt; i++) sum = sum + sc[i];
                z[r] = z[r] + sum;
            } else {
                for (int64_t i = 0; i < cnt; i++) {
                    sc[i] = ef_scale(c, sc[i]);
                    if (isfinite(sc[i])) {
                        if (sc[i] > high[r]) high[r] = sc[i];
                        if (sc[i] < light[r]) light[r] = sc[i];
                    }
                }
                for (int64_t j = lo; j < hi; j++) {
                    if (c->finite[j0 + j]) continue;
                    int infinite = 0;
                    for (int64_t y = 0; y < ny; y++) if (isinf(c->v[(j0 + j) * ny + y])) infinite = 1;
                    if (infinite && isfinite(sc[j - lo]) && sc[j - lo] < low[r]) low[r] = sc[j - lo];
                }
                double shift = 0.0;
                if (shifted) {
                    shift = m[r];
                    for (int64_t i = 0; i < cnt; i++) if (sc[i] > shift || isnan(sc[i])) shift = sc[i];
                }
                if (shift == -INFINITY) {
                    for (int64_t i = 0; i < cnt; i++) sc[i] = 0.0;
                    continue;
                }
                double rescale = exp(m[r] - shift);
                double sum = 0.0;
                int special_weights = 0;
                for (int64_t i = 0; i < cnt; i++) { sc[i] = exp(sc[i] - shift); sum = sum + sc[i]; }
                for (int64_t i = 0; i < cnt; i++) if (!isfinite(sc[i])) special_weights = 1;
                if (shifted && rescale != 1.0) {
                    overflowed |= ef_overflows(z[r], a + r * ny, special_weight[r], special_value + r * ny, ny);
                    z[r] = z[r] * rescale;
                    for (int64_t y = 0; y < ny; y++) a[r * ny + y] = a[r * ny + y] * rescale;
                }
                special_weight[r] |= special_weights;
                int special_values = 0;
                for (int64_t j = lo; j < hi; j++) if (!c->finite[j0 + j]) special_values = 1;
                if (special_values) {
                    for (int64_t j = lo; j < hi; j++) {
                        if (c->finite[j0 + j]) continue;
                        for (int64_t y = 0; y < ny; y++)
                            special_value[r * ny + y] |= !isfinite(c->v[(j0 + j) * ny + y]);
                    }
                }
                if (unnormalized) overflowed |= special_weights || special_values;
                z[r] = z[r] + sum;
                m[r] = shift;
            }
        }
        /* a += w · v over each row's allowed span, k in order. */
        for (int64_t r = 0; r < rows; r++) {
            int64_t lo = slo[r], hi = shi[r];
            if (lo >= hi) continue;
            for (int64_t y = 0; y < ny; y++) {
                double s = a[r * ny + y];
                for (int64_t j = lo; j < hi; j++) {
                    double pr = block[r * width + j] * c->v[(j0 + j) * ny + y];
                    s = s + pr;
                }
                a[r * ny + y] = s;
            }
        }
    }
    if (unnormalized) {
        for (int64_t r = 0; r < rows; r++)
            if (shifted && m[r] == -INFINITY)
                for (int64_t y = 0; y < ny; y++) a[r * ny + y] = NAN;
    } else {
        for (int64_t r = 0; r < rows; r++) {
            double *row = a + r * ny;
            overflowed |= ef_overflows(z[r], row, special_weight[r], special_value + r * ny, ny);
            for (int64_t y = 0; y < ny; y++) row[y] = row[y] / z[r];
            overflowed |= z[r] != 0.0 && ef_overflows(z[r], row, special_weight[r], special_value + r * ny, ny);
        }
    }
    for (int64_t r = 0; r < rows; r++) {
        double heaviest, lightest;
        if (map) { heaviest = high[r]; lightest = light[r]; }
        else if (shifted) { heaviest = exp(high[r] - m[r]); lightest = exp(light[r] - m[r]); }
        else { heaviest = exp(high[r]); lightest = exp(light[r]); }
        if (special_weight[r] || high[r] == -INFINITY || heaviest == 0.0) continue;
        int zp = !unnormalized;
        if (!ef_bounds_hold(heaviest, lightest, row_largest[r], row_smallest[r], terms[r], zp, z[r],
                            a + r * ny, special_value + r * ny, ny))
            overflowed = 1;
        if (low[r] != INFINITY) {
            double lw = shifted ? exp(low[r] - m[r]) : exp(low[r]);
            double normal = 2.0 * 2.2250738585072014e-308;
            int ok = lw >= normal && (!zp || lw / fabs(z[r]) >= normal);
            if (!ok) overflowed = 1;
        }
    }
    c->visited[t] = visited;
    c->overflowed[t] = (uint8_t)overflowed;
    free(m); free(z); free(block); free(special_weight); free(special_value); free(high); free(light);
    free(terms); free(row_largest); free(row_smallest); free(low); free(slo); free(shi);
}

/* Runs every X tile. Shape = {nx, ne, nj, ny, local_nx, local_nj}. Returns
 * tiles visited; *overflowed is set if any tile overflowed. */
int64_t ef_fused(const int64_t *shape, int weight_kind, int scale_kind, double scale_c, int shifted, int normalizer,
                 const ef_node *weight_nodes, int weight_n, int scores_kind, const double *q, const double *kt,
                 const ef_node *score_nodes, int score_n, int n_slots, const double *const *mats, const int *side,
                 int n_mask, const int *mask_cmp, const int64_t *mask_off, const double *v, const uint8_t *finite,
                 const double *largest, const double *smallest, double *out, int threads, int *overflowed) {
    ef_fused_ctx c;
    c.nx = shape[0]; c.ne = shape[1]; c.nj = shape[2]; c.ny = shape[3]; c.local_nx = shape[4]; c.local_nj = shape[5];
    c.weight_kind = weight_kind; c.scale_kind = scale_kind; c.scale_c = scale_c; c.shifted = shifted;
    c.normalizer = normalizer; c.weight_nodes = weight_nodes; c.weight_n = weight_n;
    c.scores_kind = scores_kind; c.q = q; c.kt = kt; c.score_nodes = score_nodes; c.score_n = score_n;
    c.n_slots = n_slots; c.mats = mats; c.side = side;
    c.n_mask = n_mask; c.mask_cmp = mask_cmp; c.mask_off = mask_off;
    c.v = v; c.finite = finite; c.largest = largest; c.smallest = smallest; c.out = out;
    int64_t tiles = (c.nx + EF_XT - 1) / EF_XT;
    c.visited = (int64_t *)calloc((size_t)(tiles + 1), sizeof(int64_t));
    c.overflowed = (uint8_t *)calloc((size_t)(tiles + 1), 1);
    ef_par_tasks(tiles, threads, ef_fused_tile, &c);
    int64_t visited = 0;
    int of = 0;
    for (int64_t t = 0; t < tiles; t++) { visited += c.visited[t]; of |= c.overflowed[t]; }
    *overflowed = of;
    free(c.visited); free(c.overflowed);
    return visited;
}
