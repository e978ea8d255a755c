/*
 * louvain_oracle.c -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
 *
 * A CPU restatement of the reference's Louvain pipeline (FedeFonto/louvain-fast-move-cuda),
 * used only as the parity checker by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline leg and its CPU reference arm. The CUDA engine never links or calls it.
 *
 * What it restates, phase by phase (file:line in the reference):
 *   level loop + stop rule        modularityAlgorithms.h:31-67 (cont = Q_end - Q_start > thr)
 *   iteration loop + stop rule    phaseOptimization.cuh:158-181 (at least one iteration,
 *                                 stop when dQ <= thr; moves of the last iteration kept)
 *   iteration 0 ("fast")          phaseOptimizationSort.cu:28-158: per-edge gain with
 *                                 self = 0, argmax per source in CSR order (strict '>',
 *                                 operators.h:30-40 GetMaxValue: first maximum wins)
 *   iteration >= 1 (SORT)         phaseOptimizationSort.cu:161-379: per-(v,c) sums of
 *                                 non-loop edge weights, self_v = w(v, comm v),
 *                                 argmax over c ascending with strict '>' (lowest c wins)
 *   iteration >= 1 (HASH)         phaseOptimizationHash.cu:23-35 + hashmap.cuh:46-73:
 *                                 own community excluded, only gain > 0, atomicMax of
 *                                 (gain bits << 32 | c): highest c wins among equal gains
 *   gain                          operatorsDelta.h:29-45: (float)((w_vc - self_v)/m
 *                                 + k_v (a_own - k_v - a_c) / (2 m m)); the subtraction
 *                                 w_vc - self_v is a float subtraction, the rest double
 *   move rule                     phaseOptimizationUpdate.cu:64 (c != comm v, gain > 0),
 *                                 :99 adds v <= c for iteration 0
 *   synchronous moves             phaseOptimizationUpdate.cu:47-115 (all gains from the
 *                                 pre-iteration state; totals += / -= k_v)
 *   active set                    phaseOptimizationUpdate.cu:117-132 (v active next iff a
 *                                 neighbour moved and now sits in another community)
 *   chunk early return            phaseOptimizationSort.cu:46-86,186-240 (edge chunks of
 *                                 STEP_ROUND ending at neighboorhood_sum[src[limit]-1];
 *                                 the first chunk with no selected edge ends the pass)
 *   modularity                    community.h:68-106: Q = I/(2m) - S/(4 m m)
 *   aggregation                   phaseAggregation.cuh:27-174: new id = (#nonempty c'<=c)-1,
 *                                 best[v0] = new(comm[best[v0]]), contraction to sorted
 *                                 (c_s, c_d, sum w) rows, k' = row sums, identity restart
 *
 * Refinement (cfg.refine = 1; no reference counterpart -- RefinePhase, phaseRefine.cuh:1-3, is
 * an empty hook). The refinement step of Leiden (Traag, Waltman, van Eck 2019, "From Louvain to
 * Leiden", Algorithm A.2 RefinePartition / MergeNodesSubset) in a greedy, pass-synchronous
 * form, run after a level's local moving:
 *   - the refined partition starts as singletons (ref[v] = v, aref[v] = k_v);
 *   - v may move iff it is still a singleton and was well connected to its community S at the
 *     start: 2m * w(v, S - v) >= k_v (K_S - k_v), K_S = a[S] (exact in 128-bit integers);
 *   - a pass evaluates, for every such v, the refined communities of its neighbours inside S
 *     with the gain and tie rule of a regular pass of the level's mode (own singleton:
 *     self = 0, a_own = k_v) and proposes the best one if its gain is > 0;
 *   - proposals are resolved from the pre-pass state: v -> t is kept unless t is a singleton
 *     that itself proposes, except that of two singletons proposing each other the higher id
 *     joins the lower; kept moves update ref, aref and the member counts;
 *   - passes repeat while the refined partition's modularity rises by more than the threshold
 *     (at most refine_passes passes when that is > 0, and the iteration limit).
 * The level is then aggregated by the refined partition, and the next level starts from
 * singletons as usual (Leiden starts it from the coarse partition; with the reference's
 * synchronous moves that start oscillates, because the pass-0 v <= c gate only breaks the
 * symmetry of a singleton start). A refined level continues iff its aggregate graph is
 * smaller (n_ref < n) and either Q rose by more than the threshold since the previous
 * level's end or n_ref < refine_tolerance * n; otherwise the run ends with the coarse
 * partition -- or, when that level ended below the previous level's end, with the previous
 * level's partition (each vertex of a level keeps its members' community of the level before,
 * `prev`), so a refined run never ends below an earlier level's end. Refined communities are
 * connected: a vertex only joins a community holding one of its neighbours that stays where
 * it is.
 *
 * Arithmetic: compiled with -ffp-contract=off so every double operation rounds once, as
 * the device code does. Weight sums are accumulated in double; with integer weights and
 * total weight below 2^32 (the reference's own u32 limit) every sum is exact, so summation
 * order cannot matter. S = sum a_c^2 is accumulated exactly in 128-bit integers for integer
 * weights. With fp32 weights (no reference counterpart) sums are double, S is a sequential
 * double sum and contracted weights are rounded to fp32 once.
 *
 * Parallelism (OpenMP) only splits work whose result does not depend on the split: the
 * per-vertex decisions of one pass, the active-set rule and exact integer reductions.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_NOMEM 2
#define ORC_ERR_RANGE 3

typedef struct {
    int32_t mode;            /* 0 = HASH rule, 1 = SORT rule (constants.h:13 order) */
    int32_t fast_first;      /* iteration 0 is the per-edge "fast" pass with v <= c */
    int32_t max_iterations;  /* EARLY_STOP_LIMIT (constants.h:16) */
    int32_t max_levels;      /* 0 = unlimited */
    double threshold;        /* MODULARITY_CONVERGED_THRESHOLD (constants.h:15) */
    int64_t chunk_edges;     /* STEP_ROUND (constants.h:18); 0 disables the emulation */
    int32_t nthreads;        /* 0 = OpenMP default */
    int32_t integer_weights; /* 1 = weights are integers (reference semantics) */
    int32_t refine;          /* 1 = refine the partition before each aggregation */
    int32_t refine_passes;   /* refinement pass limit, 0 = until converged */
    double refine_tolerance; /* a refined level continues while n_ref < tolerance * n */
} orc_config;

typedef struct {
    int32_t level, iteration, n_considered, n_moved;
    double internal, sum_a2, modularity, delta;
    int64_t n_pairs;         /* (v, c != comm v) candidate pairs of the pass */
    int64_t n_internal;      /* edge entries with comm[src] == comm[dst] after the pass */
} orc_iter_record;

typedef struct {
    orc_config cfg;
    /* current level graph */
    int64_t n, E;
    int64_t* row_ptr;
    int32_t* col;
    uint32_t* wi;   /* integer weights (integer mode) */
    float* wf;      /* fp32 weights (float mode) */
    double* k;      /* tot_weight_per_nodes */
    /* partition state */
    int32_t* comm;
    double* a;      /* communities_weight */
    uint8_t* active;
    uint8_t* moved;
    int32_t* best;  /* best_communities, one per original vertex */
    int64_t n0;
    double m;       /* total_weight, fixed at level 0 */
    double modularity, internal, sum_a2;
    int64_t n_internal_entries;
    int64_t overrun_events;  /* community.h:69,85 buffers of 2*(E/2) entries would be too
                                short: E odd and (n == E or every entry internal) */
    int64_t n_best;
    int32_t level;
    int32_t iter_in_level;
    int64_t refine_passes_run;
    int32_t* prev;  /* refined runs: each vertex's community at the end of the previous level,
                       labelled by the smallest vertex id of that community */
    /* scratch */
    int32_t* dec_c;
    float* dec_g;
    /* trace */
    orc_iter_record* trace;
    int64_t trace_len, trace_cap;
} orc_state;

static inline double wget(const orc_state* s, int64_t e) {
    return s->cfg.integer_weights ? (double)s->wi[e] : (double)s->wf[e];
}

/* operatorsDelta.h:29-45 with the reference's operand types: float w_vc, float self,
 * unsigned (here double-valued) k, double totals and total weight. */
static inline float gain_ref(float w_vc, float self_v, double k, double a_own, double a_c, double m) {
    float diff = w_vc - self_v;
    double t1 = (double)diff / m;
    double t2 = (k * ((a_own - k) - a_c)) / ((2.0 * m) * m);
    return (float)(t1 + t2);
}

static int nthreads_of(const orc_state* s) {
#ifdef _OPENMP
    return s->cfg.nthreads > 0 ? s->cfg.nthreads : omp_get_max_threads();
#else
    (void)s;
    return 1;
#endif
}


static int cmp_i32(const void* x, const void* y) {
    int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
    return (a > b) - (a < b);
}

/* ascending order: the order sort_by_key leaves (src, community) keys in */
static void sort_i32(int32_t* a, int32_t cnt) {
    if (cnt > 32) { qsort(a, (size_t)cnt, sizeof(int32_t), cmp_i32); return; }
    for (int32_t i = 1; i < cnt; i++) {
        int32_t x = a[i]; int32_t j = i - 1;
        while (j >= 0 && a[j] > x) { a[j + 1] = a[j]; j--; }
        a[j + 1] = x;
    }
}

/* threads for passes that keep an n-sized accumulator per thread: stay under a memory
 * budget (ORACLE_SCRATCH_BYTES, default 4 GiB) */
static int nthreads_for_scratch(const orc_state* s, int64_t n) {
    int nt = nthreads_of(s);
    const char* env = getenv("ORACLE_SCRATCH_BYTES");
    double budget = env ? atof(env) : 4294967296.0;
    double per = 20.0 * (double)(n > 0 ? n : 1);
    int cap = (int)(budget / per);
    if (cap < 1) cap = 1;
    return nt < cap ? nt : cap;
}

static void compute_modularity(orc_state* s) {
    /* community.h:68-106 */
    int64_t n = s->n;
    double internal = 0.0;
    if (s->cfg.integer_weights) {
        uint64_t in = 0;
        int64_t cnt = 0;
        int nt = nthreads_of(s);
        #pragma omp parallel for reduction(+:in,cnt) schedule(static) num_threads(nt)
        for (int64_t v = 0; v < n; v++) {
            uint64_t acc = 0;
            int32_t cv = s->comm[v];
            for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++)
                if (s->comm[s->col[e]] == cv) { acc += s->wi[e]; cnt++; }
            in += acc;
        }
        s->n_internal_entries = cnt;
        internal = (double)in;
        unsigned __int128 sq = 0;
        for (int64_t c = 0; c < n; c++) {
            uint64_t ac = (uint64_t)s->a[c];
            sq += (unsigned __int128)ac * ac;
        }
        s->sum_a2 = (double)sq;
    } else {
        int64_t cnt = 0;
        for (int64_t v = 0; v < n; v++) {
            int32_t cv = s->comm[v];
            for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++)
                if (s->comm[s->col[e]] == cv) { internal += s->wf[e]; cnt++; }
        }
        s->n_internal_entries = cnt;
        double sq = 0.0;
        for (int64_t c = 0; c < n; c++) sq += s->a[c] * s->a[c];
        s->sum_a2 = sq;
    }
    s->internal = internal;
    if ((s->E & 1) && (s->n == s->E || s->n_internal_entries == s->E)) s->overrun_events++;
    double m = s->m;
    s->modularity = internal / (2.0 * m) - s->sum_a2 / ((4.0 * m) * m);
}

static void level_reset(orc_state* s) {
    /* community.h:57-65 update(): identity partition, totals = k; all vertices active
     * (phaseOptimization.cuh:52) */
    for (int64_t v = 0; v < s->n; v++) {
        s->comm[v] = (int32_t)v;
        s->a[v] = s->k[v];
        s->active[v] = 1;
        s->moved[v] = 0;
    }
    s->iter_in_level = 0;
    compute_modularity(s);
}

static void free_graph(orc_state* s) {
    free(s->row_ptr); free(s->col); free(s->wi); free(s->wf); free(s->k);
    s->row_ptr = NULL; s->col = NULL; s->wi = NULL; s->wf = NULL; s->k = NULL;
}

void orc_destroy(orc_state* s) {
    if (!s) return;
    free_graph(s);
    free(s->comm); free(s->a); free(s->active); free(s->moved); free(s->best);
    free(s->dec_c); free(s->dec_g); free(s->trace); free(s->prev);
    free(s);
}

orc_state* orc_create(int64_t n, const int64_t* row_ptr, const int32_t* col, const float* w,
                      const orc_config* cfg, int32_t* err) {
    *err = ORC_OK;
    if (n <= 0 || !row_ptr || !col || !cfg) { *err = ORC_ERR_ARG; return NULL; }
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    if (!s) { *err = ORC_ERR_NOMEM; return NULL; }
    s->cfg = *cfg;
    if (w == NULL) s->cfg.integer_weights = 1;
    s->n = s->n0 = n;
    s->E = row_ptr[n];
    s->row_ptr = (int64_t*)malloc((size_t)(n + 1) * sizeof(int64_t));
    s->col = (int32_t*)malloc((size_t)(s->E > 0 ? s->E : 1) * sizeof(int32_t));
    s->k = (double*)malloc((size_t)n * sizeof(double));
    s->comm = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    s->a = (double*)malloc((size_t)n * sizeof(double));
    s->active = (uint8_t*)malloc((size_t)n);
    s->moved = (uint8_t*)malloc((size_t)n);
    s->best = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    s->dec_c = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    s->dec_g = (float*)malloc((size_t)n * sizeof(float));
    if (s->cfg.integer_weights) s->wi = (uint32_t*)malloc((size_t)(s->E > 0 ? s->E : 1) * sizeof(uint32_t));
    else s->wf = (float*)malloc((size_t)(s->E > 0 ? s->E : 1) * sizeof(float));
    if (!s->row_ptr || !s->col || !s->k || !s->comm || !s->a || !s->active || !s->moved ||
        !s->best || !s->dec_c || !s->dec_g || (!s->wi && !s->wf)) {
        orc_destroy(s); *err = ORC_ERR_NOMEM; return NULL;
    }
    memcpy(s->row_ptr, row_ptr, (size_t)(n + 1) * sizeof(int64_t));
    memcpy(s->col, col, (size_t)s->E * sizeof(int32_t));
    double total = 0.0;
    for (int64_t v = 0; v < n; v++) {
        double kv = 0.0;
        for (int64_t e = row_ptr[v]; e < row_ptr[v + 1]; e++) {
            if (col[e] < 0 || col[e] >= n) { orc_destroy(s); *err = ORC_ERR_ARG; return NULL; }
            if (s->cfg.integer_weights) {
                double x = w ? (double)w[e] : 1.0;
                if (x < 0 || x != floor(x) || x > 4294967295.0) { orc_destroy(s); *err = ORC_ERR_ARG; return NULL; }
                s->wi[e] = (uint32_t)x;
                kv += x;
            } else {
                s->wf[e] = w[e];
                kv += (double)w[e];
            }
        }
        s->k[v] = kv;
        total += kv;
        s->best[v] = (int32_t)v;
    }
    if (s->cfg.integer_weights && total >= 4294967296.0) { orc_destroy(s); *err = ORC_ERR_RANGE; return NULL; }
    /* graph.cu:81 total_weight = n_links: half the directed weight sum */
    s->m = total / 2.0;
    s->n_best = n;
    s->level = 0;
    level_reset(s);
    return s;
}

/* Vertex ranges [lo, hi) of the reference's edge chunks for the current level. */
static int64_t chunk_bounds(const orc_state* s, int64_t* lo_out, int64_t* hi_out, int64_t cap) {
    int64_t E = s->E, step = s->cfg.chunk_edges, nch = 0;
    if (step <= 0 || E <= step) {
        lo_out[0] = 0; hi_out[0] = s->n;
        return 1;
    }
    int64_t round = 0;
    while (round < E && nch < cap) {
        int64_t limit = round + step;
        if (limit >= E) {
            limit = E;
        } else {
            /* limit = neighboorhood_sum[edge_source[limit] - 1] */
            int64_t lo = 0, hi = s->n; /* find src of edge `limit` */
            while (hi - lo > 1) { int64_t mid = (lo + hi) / 2; if (s->row_ptr[mid] <= limit) lo = mid; else hi = mid; }
            int64_t srcv = lo;
            if (srcv == 0) return -1;
            limit = s->row_ptr[srcv - 1];
            if (limit <= round) return -1; /* the reference would loop forever */
        }
        int64_t vlo = 0, vhi = s->n;
        { int64_t lo = 0, hi = s->n; while (hi - lo > 1) { int64_t mid = (lo + hi) / 2; if (s->row_ptr[mid] <= round) lo = mid; else hi = mid; } vlo = lo; }
        if (limit >= E) vhi = s->n;
        else { int64_t lo = 0, hi = s->n; while (hi - lo > 1) { int64_t mid = (lo + hi) / 2; if (s->row_ptr[mid] <= limit) lo = mid; else hi = mid; } vhi = lo; }
        lo_out[nch] = vlo; hi_out[nch] = vhi; nch++;
        round = limit;
    }
    return nch;
}

static int has_selected_edge(const orc_state* s, int64_t v) {
    if (!s->active[v]) return 0;
    for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++)
        if (s->col[e] != v) return 1;
    return 0;
}

/* One optimize() + fast_move_update() + compute_modularity() of the reference.
 * Returns the number of vertices that moved. */
static int64_t optimization_step(orc_state* s) {
    int64_t n = s->n;
    const int fast = s->cfg.fast_first && s->iter_in_level == 0;
    /* phaseOptimization.cuh:135: HASH and ADAPTIVE_MEMORY use the hash rule from pass 1,
     * ADAPTIVE_SPEED after pass 4 */
    const int m_ = s->cfg.mode;
    const int hash_rule = !fast && (m_ == 0 || m_ == 3 || (m_ == 2 && s->iter_in_level > 4));
    /* which vertices does this pass consider (chunk early return) */
    int64_t v_end = n;
    int chunk_rule = (s->cfg.chunk_edges > 0) && (fast || !hash_rule);
    if (chunk_rule && s->E > s->cfg.chunk_edges) {
        int64_t cap = s->E / (s->cfg.chunk_edges > 0 ? s->cfg.chunk_edges : 1) + 8;
        int64_t* lo = (int64_t*)malloc((size_t)cap * sizeof(int64_t));
        int64_t* hi = (int64_t*)malloc((size_t)cap * sizeof(int64_t));
        int64_t nch = chunk_bounds(s, lo, hi, cap);
        for (int64_t ch = 0; ch < nch; ch++) {
            int any = 0;
            for (int64_t v = lo[ch]; v < hi[ch] && !any; v++) any = has_selected_edge(s, v);
            if (!any) { v_end = lo[ch]; break; }
        }
        free(lo); free(hi);
    }

    int64_t considered = 0, pairs = 0;
    int nt = nthreads_of(s);
    int nts = fast ? nt : nthreads_for_scratch(s, n);
    #pragma omp parallel num_threads(nts) reduction(+:considered,pairs)
    {
        double* acc = NULL;
        int32_t* stamp = NULL;
        int32_t* touched = NULL;
        if (!fast) {
            acc = (double*)malloc((size_t)n * sizeof(double));
            stamp = (int32_t*)malloc((size_t)n * sizeof(int32_t));
            touched = (int32_t*)malloc((size_t)n * sizeof(int32_t));
            for (int64_t i = 0; i < n; i++) stamp[i] = -1;
        }
        #pragma omp for schedule(dynamic, 256)
        for (int64_t v = 0; v < n; v++) {
            s->dec_c[v] = -1;
            if (v >= v_end || !has_selected_edge(s, v)) continue;
            considered++;
            int32_t cv = s->comm[v];
            double kv = s->k[v];
            double a_own = s->a[cv];
            if (fast) {
                /* per-edge gains, self = 0, first maximum in CSR order wins */
                int32_t bc = -1; float bg = 0.0f; int have = 0;
                for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++) {
                    int32_t u = s->col[e];
                    if (u == v) continue;
                    int32_t cu = s->comm[u];
                    float wf = (float)wget(s, e);
                    float g = gain_ref(wf, 0.0f, kv, a_own, s->a[cu], s->m);
                    if (!have || g > bg) { bg = g; bc = cu; have = 1; }
                }
                s->dec_c[v] = bc; s->dec_g[v] = bg;
            } else {
                int32_t nt_ = 0;
                for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++) {
                    int32_t u = s->col[e];
                    if (u == v) continue;
                    int32_t cu = s->comm[u];
                    if (stamp[cu] != (int32_t)v) { stamp[cu] = (int32_t)v; acc[cu] = 0.0; touched[nt_++] = cu; }
                    acc[cu] += wget(s, e);
                }
                sort_i32(touched, nt_);
                float self_v = (stamp[cv] == (int32_t)v) ? (float)acc[cv] : 0.0f;
                pairs += nt_ - ((stamp[cv] == (int32_t)v) ? 1 : 0);
                int32_t bc = -1; float bg = 0.0f; int have = 0;
                for (int32_t i = 0; i < nt_; i++) {
                    int32_t c = touched[i];
                    if (hash_rule && c == cv) continue;
                    float g = gain_ref((float)acc[c], self_v, kv, a_own, s->a[c], s->m);
                    if (hash_rule) {
                        if (g > 0.0f && (!have || g >= bg)) { bg = g; bc = c; have = 1; }
                    } else {
                        if (!have || g > bg) { bg = g; bc = c; have = 1; }
                    }
                }
                s->dec_c[v] = bc; s->dec_g[v] = bg;
            }
        }
        free(acc); free(stamp); free(touched);
    }

    /* update_value_kernel_* : apply every move from the pre-iteration state */
    int64_t moved = 0;
    memset(s->moved, 0, (size_t)n);
    for (int64_t v = 0; v < n; v++) {
        int32_t c = s->dec_c[v];
        if (c < 0) continue;
        if (s->comm[v] == c || !(s->dec_g[v] > 0.0f)) continue;
        if (fast && v > c) continue;
        s->a[c] += s->k[v];
        s->a[s->comm[v]] -= s->k[v];
        s->comm[v] = c;
        s->moved[v] = 1;
        moved++;
    }
    /* update_changed_kernel */
    #pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t v = 0; v < n; v++) {
        uint8_t act = 0;
        int32_t cv = s->comm[v];
        for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1] && !act; e++) {
            int32_t u = s->col[e];
            if (s->moved[u] && s->comm[u] != cv) act = 1;
        }
        s->active[v] = act;
    }
    double q_old = s->modularity;
    compute_modularity(s);
    if (s->trace_len == s->trace_cap) {
        int64_t cap = s->trace_cap ? 2 * s->trace_cap : 64;
        orc_iter_record* t = (orc_iter_record*)realloc(s->trace, (size_t)cap * sizeof(orc_iter_record));
        if (t) { s->trace = t; s->trace_cap = cap; }
    }
    if (s->trace_len < s->trace_cap) {
        orc_iter_record* r = &s->trace[s->trace_len++];
        r->level = s->level; r->iteration = s->iter_in_level;
        r->n_considered = (int32_t)considered; r->n_moved = (int32_t)moved;
        r->internal = s->internal; r->sum_a2 = s->sum_a2;
        r->modularity = s->modularity; r->delta = s->modularity - q_old;
        r->n_pairs = pairs; r->n_internal = s->n_internal_entries;
    }
    s->iter_in_level++;
    return moved;
}

/* Modularity of an arbitrary partition `part` with totals `tot` (same arithmetic as
 * compute_modularity). */
static double partition_modularity(const orc_state* s, const int32_t* part, const double* tot) {
    int64_t n = s->n;
    double internal = 0.0, sq_d = 0.0;
    if (s->cfg.integer_weights) {
        uint64_t in = 0;
        for (int64_t v = 0; v < n; v++)
            for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++)
                if (part[s->col[e]] == part[v]) in += s->wi[e];
        unsigned __int128 sq = 0;
        for (int64_t c = 0; c < n; c++) {
            uint64_t ac = (uint64_t)tot[c];
            sq += (unsigned __int128)ac * ac;
        }
        internal = (double)in;
        sq_d = (double)sq;
    } else {
        for (int64_t v = 0; v < n; v++)
            for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++)
                if (part[s->col[e]] == part[v]) internal += s->wf[e];
        for (int64_t c = 0; c < n; c++) sq_d += tot[c] * tot[c];
    }
    double m = s->m;
    return internal / (2.0 * m) - sq_d / ((4.0 * m) * m);
}

/* The refinement of the current (coarse) partition s->comm; returns the refined partition
 * (labels are vertex ids) or NULL when out of memory. Semantics in the header comment. */
static int32_t* refine_partition(orc_state* s) {
    int64_t n = s->n;
    int32_t* ref = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    int32_t* prop = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    int32_t* rsz = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    double* aref = (double*)malloc((size_t)n * sizeof(double));
    uint8_t* wc = (uint8_t*)malloc((size_t)n);
    uint8_t* keep = (uint8_t*)malloc((size_t)n);
    if (!ref || !prop || !rsz || !aref || !wc || !keep) {
        free(ref); free(prop); free(rsz); free(aref); free(wc); free(keep);
        return NULL;
    }
    const double two_m = 2.0 * s->m;
    for (int64_t v = 0; v < n; v++) {
        const int32_t cv = s->comm[v];
        if (s->cfg.integer_weights) {
            uint64_t wv = 0;
            for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++) {
                int32_t u = s->col[e];
                if (u != v && s->comm[u] == cv) wv += s->wi[e];
            }
            const uint64_t kv = (uint64_t)s->k[v], K = (uint64_t)s->a[cv];
            wc[v] = (unsigned __int128)(uint64_t)two_m * wv >= (unsigned __int128)kv * (K - kv);
        } else {
            double wv = 0.0;
            for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++) {
                int32_t u = s->col[e];
                if (u != v && s->comm[u] == cv) wv += s->wf[e];
            }
            wc[v] = two_m * wv >= s->k[v] * (s->a[cv] - s->k[v]);
        }
        ref[v] = (int32_t)v;
        aref[v] = s->k[v];
        rsz[v] = 1;
    }
    double q = partition_modularity(s, ref, aref);
    const int m_ = s->cfg.mode;
    for (int32_t p = 0;;) {
        /* the level's tie rule for a regular pass with index p (phaseOptimization.cuh:135) */
        const int hash_rule = m_ == 0 || m_ == 3 || (m_ == 2 && p > 4);
        int nts = nthreads_for_scratch(s, n);
        #pragma omp parallel num_threads(nts)
        {
            double* acc = (double*)malloc((size_t)n * sizeof(double));
            int32_t* stamp = (int32_t*)malloc((size_t)n * sizeof(int32_t));
            int32_t* touched = (int32_t*)malloc((size_t)n * sizeof(int32_t));
            for (int64_t i = 0; i < n; i++) stamp[i] = -1;
            #pragma omp for schedule(dynamic, 256)
            for (int64_t v = 0; v < n; v++) {
                prop[v] = ref[v];
                if (!(ref[v] == (int32_t)v && rsz[v] == 1 && wc[v])) continue;
                const int32_t cv = s->comm[v];
                int32_t nt_ = 0;
                for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++) {
                    int32_t u = s->col[e];
                    if (u == v || s->comm[u] != cv) continue;
                    int32_t r = ref[u];
                    if (stamp[r] != (int32_t)v) { stamp[r] = (int32_t)v; acc[r] = 0.0; touched[nt_++] = r; }
                    acc[r] += wget(s, e);
                }
                if (nt_ == 0) continue;
                sort_i32(touched, nt_);
                const int32_t own = ref[v];
                float self_v = (stamp[own] == (int32_t)v) ? (float)acc[own] : 0.0f;
                double kv = s->k[v], a_own = aref[own];
                int32_t bc = -1; float bg = 0.0f; int have = 0;
                for (int32_t i = 0; i < nt_; i++) {
                    int32_t c = touched[i];
                    if (hash_rule && c == own) continue;
                    float g = gain_ref((float)acc[c], self_v, kv, a_own, aref[c], s->m);
                    if (hash_rule) {
                        if (g > 0.0f && (!have || g >= bg)) { bg = g; bc = c; have = 1; }
                    } else {
                        if (!have || g > bg) { bg = g; bc = c; have = 1; }
                    }
                }
                if (bc >= 0 && bc != own && bg > 0.0f) prop[v] = bc;
            }
            free(acc); free(stamp); free(touched);
        }
        /* resolution from the pre-pass state, then the kept moves */
        for (int64_t v = 0; v < n; v++) {
            keep[v] = 0;
            if (prop[v] == ref[v]) continue;
            const int32_t t = prop[v];
            const int t_proposes = ref[t] == t && rsz[t] == 1 && prop[t] != t;
            keep[v] = !t_proposes || (prop[t] == (int32_t)v && t < (int32_t)v);
        }
        for (int64_t v = 0; v < n; v++) {
            if (!keep[v]) continue;
            const int32_t t = prop[v], o = ref[v];
            aref[t] += s->k[v];
            aref[o] -= s->k[v];
            ref[v] = t;
            rsz[t]++;
            rsz[o]--;
        }
        const double qn = partition_modularity(s, ref, aref);
        const double dq = qn - q;
        q = qn;
        p++;
        s->refine_passes_run++;
        if (!(dq > s->cfg.threshold) || p > s->cfg.max_iterations ||
            (s->cfg.refine_passes > 0 && p >= s->cfg.refine_passes))
            break;
    }
    free(prop); free(rsz); free(aref); free(wc); free(keep);
    return ref;
}

/* OptimizationPhase::run (phaseOptimization.cuh:158-206) */
int32_t orc_optimization_run(orc_state* s) {
    double delta;
    int32_t it = 0;
    do {
        double old = s->modularity;
        optimization_step(s);
        it++;
        delta = s->modularity - old;
    } while (it <= s->cfg.max_iterations && delta > s->cfg.threshold);
    return it;
}

int32_t orc_optimization_step(orc_state* s, double* delta) {
    double old = s->modularity;
    int64_t moved = optimization_step(s);
    if (delta) *delta = s->modularity - old;
    return (int32_t)moved;
}

/* AggregationPhase::run (phaseAggregation.cuh:19-190). A refined run passes its refined
 * partition in `ref` (taken over and freed): the level is aggregated by it. */
static int32_t aggregate_by(orc_state* s, int32_t aggregate, int32_t* ref) {
    int64_t n = s->n;
    if (!aggregate) { free(ref); ref = NULL; }
    const int32_t* part = ref ? ref : s->comm;
    int32_t* map = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    if (!map) { free(ref); return ORC_ERR_NOMEM; }
    int32_t run = 0;
    if (s->cfg.refine) {
        /* nonempty communities: labels with a member */
        for (int64_t c = 0; c < n; c++) map[c] = 0;
        for (int64_t v = 0; v < n; v++) map[part[v]] = 1;
        for (int64_t c = 0; c < n; c++) { run += map[c]; map[c] = run; }
    } else {
        for (int64_t c = 0; c < n; c++) { run += (s->a[c] > 0) ? 1 : 0; map[c] = run; }
    }
    /* community.h:48-55 update_best */
    for (int64_t v = 0; v < s->n0; v++) {
        int32_t b = s->best[v];
        if (b >= 0 && b < n) s->best[v] = map[part[b]] - 1;
    }
    s->n_best = run;
    if (!aggregate) { free(map); return ORC_OK; }

    int64_t n2 = run;
    /* bucket vertices by new community */
    int64_t* mptr = (int64_t*)calloc((size_t)n2 + 1, sizeof(int64_t));
    int32_t* members = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    int32_t* newc = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    if (!mptr || !members || !newc) { free(map); free(mptr); free(members); free(newc); free(ref); return ORC_ERR_NOMEM; }
    for (int64_t v = 0; v < n; v++) { newc[v] = map[part[v]] - 1; mptr[newc[v] + 1]++; }
    for (int64_t c = 0; c < n2; c++) mptr[c + 1] += mptr[c];
    {
        int64_t* cur = (int64_t*)malloc((size_t)n2 * sizeof(int64_t));
        memcpy(cur, mptr, (size_t)n2 * sizeof(int64_t));
        for (int64_t v = 0; v < n; v++) members[cur[newc[v]]++] = (int32_t)v;
        free(cur);
    }
    int64_t* cnt = (int64_t*)calloc((size_t)n2 + 1, sizeof(int64_t));
    int nt = nthreads_for_scratch(s, n2);
    /* pass 1: distinct destinations per new row; pass 2: fill sorted rows */
    int64_t* row2 = (int64_t*)calloc((size_t)n2 + 1, sizeof(int64_t));
    int32_t* col2 = NULL; uint32_t* wi2 = NULL; float* wf2 = NULL; double* k2 = NULL;
    int failed = 0;
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            for (int64_t c = 0; c < n2; c++) row2[c + 1] = row2[c] + cnt[c];
            int64_t E2 = row2[n2];
            col2 = (int32_t*)malloc((size_t)(E2 > 0 ? E2 : 1) * sizeof(int32_t));
            if (s->cfg.integer_weights) wi2 = (uint32_t*)malloc((size_t)(E2 > 0 ? E2 : 1) * sizeof(uint32_t));
            else wf2 = (float*)malloc((size_t)(E2 > 0 ? E2 : 1) * sizeof(float));
            k2 = (double*)malloc((size_t)n2 * sizeof(double));
            if (!col2 || (!wi2 && !wf2) || !k2) { failed = 1; break; }
        }
        #pragma omp parallel num_threads(nt)
        {
            double* acc = (double*)malloc((size_t)n2 * sizeof(double));
            int32_t* stamp = (int32_t*)malloc((size_t)n2 * sizeof(int32_t));
            int32_t* touched = (int32_t*)malloc((size_t)n2 * sizeof(int32_t));
            for (int64_t i = 0; i < n2; i++) stamp[i] = -1;
            #pragma omp for schedule(dynamic, 64)
            for (int64_t c = 0; c < n2; c++) {
                int32_t ntc = 0;
                for (int64_t i = mptr[c]; i < mptr[c + 1]; i++) {
                    int32_t v = members[i];
                    for (int64_t e = s->row_ptr[v]; e < s->row_ptr[v + 1]; e++) {
                        int32_t d = newc[s->col[e]];
                        if (stamp[d] != (int32_t)c) { stamp[d] = (int32_t)c; acc[d] = 0.0; touched[ntc++] = d; }
                        acc[d] += wget(s, e);
                    }
                }
                if (pass == 0) { cnt[c] = ntc; continue; }
                sort_i32(touched, ntc); /* sort_by_key on (src, dst) */
                double ksum = 0.0;
                int64_t base = row2[c];
                for (int32_t i = 0; i < ntc; i++) {
                    int32_t d = touched[i];
                    col2[base + i] = d;
                    if (s->cfg.integer_weights) { wi2[base + i] = (uint32_t)acc[d]; ksum += (double)(uint32_t)acc[d]; }
                    else { float f = (float)acc[d]; wf2[base + i] = f; ksum += (double)f; }
                }
                k2[c] = ksum;
            }
            free(acc); free(stamp); free(touched);
        }
    }
    /* refined: each new vertex remembers its members' coarse community */
    int32_t* prev = NULL;
    if (ref && !failed) {
        int32_t* lab = (int32_t*)malloc((size_t)n * sizeof(int32_t));
        prev = (int32_t*)malloc((size_t)(n2 > 0 ? n2 : 1) * sizeof(int32_t));
        if (!lab || !prev) {
            failed = 1;
            free(prev);
            prev = NULL;
        } else {
            for (int64_t c = 0; c < n; c++) lab[c] = INT32_MAX;
            for (int64_t v = 0; v < n; v++)
                if (newc[v] < lab[s->comm[v]]) lab[s->comm[v]] = newc[v];
            for (int64_t v = 0; v < n; v++) prev[newc[v]] = lab[s->comm[v]];
        }
        free(lab);
    }
    free(map); free(mptr); free(members); free(newc); free(cnt); free(ref);
    if (failed) free(prev);
    if (failed) { free(row2); free(col2); free(wi2); free(wf2); free(k2); return ORC_ERR_NOMEM; }
    free_graph(s);
    s->row_ptr = row2; s->col = col2; s->wi = wi2; s->wf = wf2; s->k = k2;
    s->n = n2; s->E = row2[n2];
    s->level++;
    level_reset(s);
    if (prev) {
        free(s->prev);
        s->prev = prev;
    }
    return ORC_OK;
}

int32_t orc_aggregation_run(orc_state* s, int32_t aggregate) {
    int32_t* ref = NULL;
    if (aggregate && s->cfg.refine) {
        ref = refine_partition(s);
        if (!ref) return ORC_ERR_NOMEM;
    }
    return aggregate_by(s, aggregate, ref);
}

/* ModularityAlgorithms::modularity_routine (modularityAlgorithms.h:14-81); the refined
 * continuation rule is in the header comment. */
int32_t orc_louvain(orc_state* s) {
    int32_t levels = 0;
    int cont;
    double prev_end = 0.0;
    do {
        double old = s->modularity;
        if (s->cfg.refine && levels > 0) old = prev_end;
        orc_optimization_run(s);
        cont = (s->modularity - old) > s->cfg.threshold;
        prev_end = s->modularity;
        levels++;
        const int last = s->cfg.max_levels > 0 && levels >= s->cfg.max_levels;
        int32_t* ref = NULL;
        if (s->cfg.refine && !last) {
            ref = refine_partition(s);
            if (!ref) return -ORC_ERR_NOMEM;
            int64_t labels = 0;  /* refined communities: labels still held by their vertex */
            for (int64_t v = 0; v < s->n; v++) labels += ref[v] == (int32_t)v ? 1 : 0;
            cont = labels < s->n &&
                   (cont || (double)labels < s->cfg.refine_tolerance * (double)s->n);
        }
        if (last) cont = 0;
        if (s->cfg.refine && !cont && s->level > 0 && s->prev && s->modularity < old) {
            /* the last level ended below the previous one: keep the previous partition */
            memcpy(s->comm, s->prev, (size_t)s->n * sizeof(int32_t));
            s->modularity = old;
        }
        int32_t rc = aggregate_by(s, cont, ref);
        if (rc != ORC_OK) return -rc;
    } while (cont);
    return levels;
}

/* ---- accessors -------------------------------------------------------------------- */
int64_t orc_n(const orc_state* s) { return s->n; }
int64_t orc_E(const orc_state* s) { return s->E; }
int64_t orc_n_best(const orc_state* s) { return s->n_best; }
int64_t orc_overrun_events(const orc_state* s) { return s->overrun_events; }
int32_t orc_level(const orc_state* s) { return s->level; }
double orc_modularity(const orc_state* s) { return s->modularity; }
double orc_internal(const orc_state* s) { return s->internal; }
double orc_sum_a2(const orc_state* s) { return s->sum_a2; }
double orc_total_weight(const orc_state* s) { return s->m; }
void orc_get_best(const orc_state* s, int32_t* out) { memcpy(out, s->best, (size_t)s->n0 * sizeof(int32_t)); }
void orc_get_comm(const orc_state* s, int32_t* out) { memcpy(out, s->comm, (size_t)s->n * sizeof(int32_t)); }
void orc_get_totals(const orc_state* s, double* out) { memcpy(out, s->a, (size_t)s->n * sizeof(double)); }
void orc_get_k(const orc_state* s, double* out) { memcpy(out, s->k, (size_t)s->n * sizeof(double)); }
void orc_get_graph(const orc_state* s, int64_t* row_ptr, int32_t* col, double* w) {
    memcpy(row_ptr, s->row_ptr, (size_t)(s->n + 1) * sizeof(int64_t));
    memcpy(col, s->col, (size_t)s->E * sizeof(int32_t));
    for (int64_t e = 0; e < s->E; e++) w[e] = wget(s, e);
}
int64_t orc_trace_len(const orc_state* s) { return s->trace_len; }
void orc_get_trace(const orc_state* s, orc_iter_record* out) {
    memcpy(out, s->trace, (size_t)s->trace_len * sizeof(orc_iter_record));
}
int32_t orc_record_size(void) { return (int32_t)sizeof(orc_iter_record); }
int64_t orc_refine_passes(const orc_state* s) { return s->refine_passes_run; }
