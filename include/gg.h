/*
 * gg.h -- C ABI of the B200 ASPL/diameter engine (libggb200.so).
 *
 * The engine computes, for a Graph Golf candidate graph, the exact all-pairs
 * shortest-path total and the diameter by a bit-parallel BFS on the GPU
 * (one bit per (source, vertex) pair, one BFS level per grid-wide step).
 *
 * Two layers:
 *  1. Calculator entry points that mirror the reference calculators one for
 *     one -- same constructor arguments, same packed edge tables the reference
 *     builds before its cudaMemcpy, same return values and sentinels:
 *       gg_graph_*   <- graphgolf::cudaASPLgraph   (cudacode/cudaASPLgraph.hpp:14-18)
 *       gg_conv_*    <- graphgolf::cudaASPLconv    (cudacode/cudaASPLconv.hpp:16-22)
 *       gg_piece_*   <- graphgolf::cudaASPLpiece   (cudacode/cudaASPLpiece.hpp:16-20)
 *       gg_box_*     <- graphgolf::cudaASPLbox     (cudacode/cudaASPLbox.hpp:16-20)
 *       gg_beamer_*  <- graphgolf::cudaASPLbeamer  (cudacode/cudaASPLbeamer.hpp:12-16)
 *     The C++ classes themselves are provided by libgg_refshim.so, which
 *     defines the reference member functions on top of these calls.
 *  2. gg_eval / gg_eval_device: the raw engine call returning exact counts
 *     (total distance, reached pairs, levels, WVC) with no sentinel folding.
 *
 * Conventions: every call returns a gg_status; GG_OK means the outputs are
 * valid.  All calls are blocking (the result is on the host when they return).
 * An engine handle must not be used by two host threads at once.  Pointers are
 * host pointers unless the name says device.
 */
#ifndef GG_H_
#define GG_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GG_ABI_VERSION 1

typedef struct gg_engine gg_engine;

typedef enum gg_status {
    GG_OK = 0,
    GG_BAD_ARG = 1,        /* argument outside the documented domain */
    GG_CUDA_ERROR = 2,     /* a CUDA runtime call failed (see gg_last_error) */
    GG_TIMEOUT = 3,        /* a bounded in-kernel wait gave up; the context stays usable */
    GG_OUT_OF_MEMORY = 4,  /* device or pinned allocation failed */
    GG_NO_DEVICE = 5       /* no CUDA device / the requested device does not exist */
} gg_status;

/* Exact outcome of one engine evaluation over the engine's sources. */
typedef struct gg_result {
    uint64_t total;      /* sum over levels L=1..levels of L * (#pairs first reached at L) */
    uint64_t reached;    /* (source, vertex) pairs reached, each source itself included */
    uint64_t pairs;      /* n_sources * n_vertices: the value `reached` has when connected */
    uint64_t scale;      /* N / M (integer division) multiplier of the lifted forms, 1 for graphs */
    int32_t levels;      /* last level that found new pairs (max eccentricity within components) */
    int32_t capped;      /* 1 if the BFS stopped at max_levels while level max_levels still found pairs */
    int32_t connected;   /* 1 if not capped and reached == pairs */
    int32_t wvc;         /* lane-aggregated completion count at the last level (want_wvc), else -1 */
    int32_t n_sources;   /* sources evaluated */
    int32_t batches;     /* source batches the engine ran */
    int32_t level_steps; /* BFS levels executed, summed over batches (the empty last level included) */
    int32_t reserved;
} gg_result;

/* Options for gg_eval; pass NULL for the defaults (all sources, no level cap). */
typedef struct gg_eval_opts {
    int32_t max_levels;       /* stop after this many levels; 0 = run to completion */
    int32_t src_begin;        /* source index range [src_begin, src_end); 0,0 = all */
    int32_t src_end;
    int32_t want_wvc;         /* track the per-level AND of the visited words (cudaASPLconv.cu:258-285) */
    uint64_t *level_counts;   /* optional host array [max_levels+1] (or [n_vertices] if uncapped):
                                 pairs first reached at each level, summed over batches */
    uint64_t *level_ns;       /* optional host array [max_levels+1]: device clock (ns) at the
                                 end of each level of the first source batch, [0] = start of
                                 level 1; entries past the last level are 0 */
} gg_eval_opts;

/* ---- calculator: plain graph (cudaASPLgraph) ------------------------------
 * adj: N * degree_max int32, row v = neighbours of v, unused slots padded with
 * v itself (self loops), exactly the table cudaASPLgraph.cu:144-153 builds.
 * calc -> (diameter, total over ordered pairs); (-1,-1) disconnected,
 * (-2,-2) if a level loop reaches step 199 (cudaASPLgraph.cu:179-190). */
gg_status gg_graph_create(int N, int degree_max, int device, gg_engine **out);
gg_status gg_graph_calc(gg_engine *e, const int32_t *adj, int *diameter, int64_t *total);

/* ---- calculator: cyclic lift "part" (cudaASPLconv) ------------------------
 * diffs: M * degree int32, row i = the diffs of orbit vertex i (padding 0),
 * exactly cudaASPLconv.cu:199-201.  Vertex v has neighbours (v + diffs[v%M]) mod N;
 * BFS runs from the M vertices 0..M-1 and the total is scaled by N/M. */
gg_status gg_conv_create(int N, int M, int degree, int device, gg_engine **out);
/* ASPL only; 1e9 if disconnected (cudaASPLconv.cu:151-196). */
gg_status gg_conv_calc(gg_engine *e, const int32_t *diffs, double *aspl);
/* (diameter, ASPL); (1e8, 1e8) if disconnected; diameter 1e8 with the ASPL of
 * levels 1..99 if the level loop ends at step 99 (cudaASPLconv.cu:197-243). */
gg_status gg_conv_diameter_aspl(gg_engine *e, const int32_t *diffs, int *diameter, double *aspl);
/* (WVC, diameter, ASPL); (1e8, 1e8, 1e8) if disconnected or step 100 still
 * finds pairs (cudaASPLconv.cu:244-308). */
gg_status gg_conv_wvc_diameter_aspl(gg_engine *e, const int32_t *diffs, int *wvc, int *diameter,
                                    double *aspl);

/* ---- calculator: 2-D torus lift "piece" (cudaASPLpiece) -------------------
 * vals: Mx*My * degree * 2 int32 (dx,dy), padding (0,0) (cudaASPLpiece.cu:166-176).
 * Sources = corner tile x<Mx, y<My; same return convention as gg_conv_diameter_aspl. */
gg_status gg_piece_create(int Nx, int Ny, int Mx, int My, int degree, int device, gg_engine **out);
gg_status gg_piece_diameter_aspl(gg_engine *e, const int32_t *vals, int *diameter, double *aspl);

/* ---- calculator: 3-D torus lift "box" (cudaASPLbox) -----------------------
 * vals: Mx*My*Mz * degree * 3 int32 (dx,dy,dz), padding (0,0,0) (cudaASPLbox.cu:170-184). */
gg_status gg_box_create(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, int device,
                        gg_engine **out);
gg_status gg_box_diameter_aspl(gg_engine *e, const int32_t *vals, int *diameter, double *aspl);

/* ---- calculator: fixed-depth pull BFS (cudaASPLbeamer) --------------------
 * Same diff table as gg_conv_*.  Reproduces cudaASPLbeamer.cu:7-84: 1e8 if
 * `regular` is 0 (:72); otherwise the pairs found within 7 levels over the
 * kernel's fixed 10^6-row scan (rows v >= N pull from (v + diff) mod N), scaled
 * by N/M, with no connectivity test.  N must be <= 10^6 (the reference's
 * bitset size). */
gg_status gg_beamer_create(int N, int M, int degree, int device, gg_engine **out);
gg_status gg_beamer_calc(gg_engine *e, const int32_t *diffs, int regular, double *aspl);

/* ---- raw engine ----------------------------------------------------------- */
/* table: the form's packed table (as for the calculator calls above). */
gg_status gg_eval(gg_engine *e, const int32_t *table, const gg_eval_opts *opts, gg_result *out);
/* Same, with the table already in device memory; `stream` (a cudaStream_t, or
 * NULL for the engine's own stream) orders the work after the caller's. */
gg_status gg_eval_device(gg_engine *e, const int32_t *d_table, const gg_eval_opts *opts,
                         gg_result *out, void *stream);

/* Milliseconds the BFS kernels of the last evaluation took on the device
 * (CUDA events on the engine stream, expansion included). */
gg_status gg_last_device_ms(gg_engine *e, double *ms);
/* Kernel launches issued by the last evaluation. */
gg_status gg_last_launches(gg_engine *e, int *launches);
/* Device clock (ns, %globaltimer) at the start and at the end of each source batch
 * of the last evaluation: ns[2*b], ns[2*b+1] for b < min(n, batches). */
gg_status gg_last_batch_ns(gg_engine *e, uint64_t *ns, int n);
/* Bytes the last evaluation copied host->device and device->host. */
gg_status gg_last_transfer_bytes(gg_engine *e, uint64_t *h2d, uint64_t *d2h);

/* Tuning: source-batch width in bits (multiple of 128; 0 = automatic). */
gg_status gg_set_batch_sources(gg_engine *e, int sources);
/* Autotuner: times `trials` evaluations of `table` for each candidate launch shape
 * -- source-batch width (fractions and multiples of the L2-resident width, and all
 * sources at once) x resident blocks per SM (as many as fit, one and two fewer) x
 * the walk pass (automatic depth, or off) -- keeps the fastest in this engine's
 * plan and records it in the tuning cache (see gg_set_tune_cache) for engines of the
 * same form, size, degree and source count on the same kind of GPU, in this process
 * and later ones.  best_sources / best_ms may be NULL. */
gg_status gg_autotune(gg_engine *e, const int32_t *table, int trials, int *best_sources,
                      double *best_ms);
/* The engine's current plan: sources per batch, resident blocks per SM, levels the
 * walk pass computes (0: none).  Any output may be NULL. */
gg_status gg_engine_plan(gg_engine *e, int *batch_sources, int *blocks_per_sm, int *walk_levels);
/* Tuning cache file (no reference counterpart): tuned launch shapes of every
 * evaluator (gg_autotune, gg_batch_autotune, gg_lift_autotune), one line per
 * (GPU name and SM count, evaluator, shape), read when an evaluator plans and
 * rewritten (atomically) when a tuner records a shape.  Default: GG_TUNE_CACHE
 * ("off": none), else $XDG_CACHE_HOME/graphgolf-b200/tune.tsv or
 * ~/.cache/graphgolf-b200/tune.tsv.  path NULL or "": keep tuned shapes in this
 * process only. */
gg_status gg_set_tune_cache(const char *path);
/* Bounded-wait limit of the in-kernel grid barrier, in milliseconds. */
gg_status gg_set_wait_limit_ms(gg_engine *e, int ms);

/* Gather-rate microbenchmark (no reference counterpart): the access pattern of a
 * dense BFS level and nothing else.  For `rows` rows of 512 bytes each (32 x 16
 * bytes, one warp per row), Y[v] = OR over `degree` random rows of X, masked
 * with Y0[v]: degree + 1 row reads and one row write per row.  Returns the best of
 * `iters` passes as GB/s of those bytes (plus the index table) and its time.
 * With rows = 65536 the three arrays (96 MiB) sit in the L2: that rate is the
 * ceiling of a dense level of a 4096-source batch on n = 65536. */
gg_status gg_gather_peak(int device, int rows, int degree, int iters, double *gbs, double *ms_per_pass);

/* Level-loop microbenchmark (no reference counterpart): the dense level loop of
 * bfs_batch_kernel outside the engine.  One cooperative launch runs `levels`
 * levels over `rows` rows of `chunks` x 16 bytes (chunks 32: 4096 sources a
 * batch, 16: 2048; two such arrays ping-ponged): each row ORs 8 neighbour rows
 * (8 random permutations, so every row is gathered 8 times a level), writes the
 * result, its popcount, flag and not-full words; the engine's grid barrier ends
 * each level.  variant 0 gathers into registers as the engine does; variant 1
 * also keeps a second row in flight a warp through cp.async into shared memory.
 * Returns the best of 4 launches' mean time a level (device timestamps, levels
 * 10.. of each launch) in microseconds.  64 <= rows <= 262144, 12 <= levels <=
 * 1024. */
gg_status gg_level_probe(int device, int rows, int chunks, int levels, int variant, double *us_per_level);

gg_status gg_destroy(gg_engine *e);

/* ---- evaluation without device allocation --------------------------------
 * No counterpart in the reference (its calculators always cudaMalloc their
 * bitsets in the constructor).  For callers that cannot allocate device memory:
 * a host whose GPU memory is all owned by another framework's pool, or a search
 * loop that cannot afford the device-wide synchronisation cudaFree implies.
 * The caller passes the inputs and outputs as device pointers:
 *   d_adj            N * degree int32 pull adjacency (entries in [0, N); pad with v itself),
 *   d_level_counts   max_levels + 1 uint64: on return, [L] = ordered pairs first
 *                    reached at BFS level L over all N sources ([0] = N); levels past
 *                    the last non-empty one are 0.  The diameter is the last L with a
 *                    nonzero count; the total distance is sum L * [L]; the graph is
 *                    connected when sum [L] == N*N.
 * Working memory is one fixed device array of GG_NOALLOC_SCRATCH_BYTES compiled into
 * the library, held by every GPU that loads it until the process exits.  N must be
 * small enough for one batch of N sources to fit in it (N <= 4096 always fits);
 * larger N returns GG_BAD_ARG.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  Calls share the array: calls whose GPU work
 * overlaps race and give undefined results.  Blocking; runs on `stream` (a
 * cudaStream_t, NULL = legacy default stream) of the current device.  Calls no
 * cudaMalloc/cudaFree. */
#define GG_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
gg_status gg_graph_eval_noalloc(const int32_t *d_adj, int N, int degree, int max_levels,
                                uint64_t *d_level_counts, void *stream);

/* ---- batched candidate evaluation (no reference counterpart) -------------
 * Replaces the reference's propose -> diameterASPL -> accept loop, which scores
 * one candidate per call (cppcode/annealing.cpp:397-403), with one launch that
 * scores thousands: every candidate is a registered base graph plus one 2-opt
 * edit (cppcode/annealing.cpp:140-197 proposes the same move).  Each candidate
 * gets the exact all-pairs total and diameter of its own graph.
 * Base graphs are plain regular graphs with fewer than 65536 vertices. */
typedef struct gg_batch gg_batch;

/* 2-opt edit of base graph `base`: remove edges (a,b) and (c,d); add (a,c),(b,d)
 * when mode == 0, or (a,d),(b,c) when mode == 1.  a < 0 means "no edit" (the base
 * itself).  In each of the four rows the first occurrence of the removed
 * neighbour is replaced. */
typedef struct gg_swap {
    int32_t base;
    int32_t a, b, c, d;
    int32_t mode;
} gg_swap;

typedef struct gg_cand_result {
    uint64_t total;       /* sum of distances over reached ordered pairs */
    uint64_t reached;     /* ordered pairs reached (n*n when connected) */
    int32_t levels;       /* eccentricity maximum = diameter when connected */
    int32_t connected;    /* reached == n*n */
} gg_cand_result;

gg_status gg_batch_create(int device, gg_batch **out);
/* Register a base graph: adj is n*degree int32 (simple, regular). */
gg_status gg_batch_add_base(gg_batch *b, int n, int degree, const int32_t *adj, int *base_id);
/* Replace a registered base graph's adjacency (same n and degree), e.g. after an
 * annealer accepted a move. */
gg_status gg_batch_set_base(gg_batch *b, int base_id, const int32_t *adj);
/* Source bits per shared-memory task for a base (128 * 2^k). */
gg_status gg_batch_set_chunk(gg_batch *b, int base_id, int sources);
/* Current source bits per task of a base. */
gg_status gg_batch_chunk(gg_batch *b, int base_id, int *sources);
/* Autotuner: for each base the candidates use, times `trials` launches of the
 * candidates with each chunk width that fits (the other bases fixed), keeps the
 * fastest and records it in the tuning cache (gg_set_tune_cache) for bases of the
 * same size and degree added later, in this process and later ones on the same
 * kind of GPU.  best_ms (may be NULL) = the fastest launch. */
gg_status gg_batch_autotune(gg_batch *b, int n_cand, const gg_swap *cands, int trials, double *best_ms);
/* Host arrays in and out; blocking.  The launch for a given candidate count is
 * captured once in a CUDA graph and replayed. */
gg_status gg_batch_eval(gg_batch *b, int n_cand, const gg_swap *cands, gg_cand_result *out);
/* Device arrays in and out, ordered on `stream` (NULL = the batch's stream); returns
 * after enqueueing.  The caller synchronises before reading `d_out`.
 * Preconditions: d_cands and d_out hold n_cand records.  The candidates are checked
 * on the device before anything is read through them (base registered, a..d inside
 * the base's vertex range and distinct, mode 0 or 1; a < 0 = the base itself): if
 * one fails, the launch scores nothing, every d_out record has levels = -1, and
 * gg_batch_device_status reports GG_BAD_ARG. */
gg_status gg_batch_eval_device(gg_batch *b, int n_cand, const gg_swap *d_cands,
                               gg_cand_result *d_out, void *stream);
/* Waits for `stream` (NULL = the batch's stream) and returns GG_BAD_ARG if the last
 * launch's device-side candidate check failed, else GG_OK; *first_bad (may be NULL) =
 * the lowest rejected candidate index, or -1. */
gg_status gg_batch_device_status(gg_batch *b, void *stream, int *first_bad);
/* Per-vertex distance histogram of a base graph: hist[v*K + k] = number of
 * vertices at distance k+1 from v, k < K (the per-row popcounts of BFS levels
 * 1..K).  hist: host array n*K. */
gg_status gg_batch_vertex_hist(gg_batch *b, int base_id, int K, uint32_t *hist);
/* Device milliseconds of the last evaluation's launch (CUDA events). */
gg_status gg_batch_last_ms(gg_batch *b, double *ms);
gg_status gg_batch_destroy(gg_batch *b);

/* ---- Incremental evaluation of 2-opt moves (no reference counterpart) ----------
 * For one current plain graph (n*degree, symmetric), a move's exact result is
 * computed by searching again only from the sources whose distances can change:
 * the full evaluation of the current graph also stores its distance matrix as 4
 * bit-planes (4*n*n/8 bytes on the device), from which a per-source test picks the
 * sources a removed edge or an added edge can affect (about 30 % of them for a
 * random 2-opt on a random regular graph).  Exact when the current graph is
 * connected with diameter <= 15; otherwise each call evaluates the moved graph in
 * full.  Plays the role of the per-proposal calculator call of the reference
 * annealers (cppcode/annealing.cpp:403-404) for large n. */
typedef struct gg_inc gg_inc;
gg_status gg_inc_create(int n, int degree, int device, gg_inc **out);
/* Make adj the current graph (full evaluation; r may be NULL). */
gg_status gg_inc_set_graph(gg_inc *h, const int32_t *adj, gg_result *r);
/* Exact counts of the current graph with move s applied (s->base is ignored);
 * *affected = sources searched again (may be NULL).  The current graph is kept. */
gg_status gg_inc_eval(gg_inc *h, const gg_swap *s, gg_cand_result *out, int *affected);
/* Apply move s to the current graph (full evaluation; r may be NULL). */
gg_status gg_inc_commit(gg_inc *h, const gg_swap *s, gg_result *r);
gg_status gg_inc_destroy(gg_inc *h);

/* ---- batched evaluation of lifted candidates (no reference counterpart) -----
 * The reference's annealers on the lifted forms propose one edit of the diff
 * table at a time and score it with one calculator call: cyclic lifts ("part",
 * cppcode/annealing.cpp:112-197 proposes, :403 scores with
 * cudaASPLconv::diameterASPL), 2-D torus lifts ("piece",
 * cppcode/pieceannealing.cpp:113-204 with cudaASPLpiece) and 3-D torus lifts
 * ("box", cppcode/boxHillClimb.cpp:113-220 with cudaASPLbox).  Here one
 * cooperative launch scores a whole population of edits of one base table: every
 * candidate is the base diff table (the table of gg_conv_* / gg_piece_* /
 * gg_box_*) with up to 4 slots replaced, and gets the exact counts of its own
 * lift with BFS from the orbit representatives (vertices 0..M-1 of a part, the
 * corner tile of a piece or box).  Each lifted size must be a multiple of the
 * matching orbit size. */
typedef struct gg_lift gg_lift;

/* Slots (row[j], slot[j]) of the base table take the diff diff[j], j < count
 * (0 <= count <= 4; count 0 is the base itself).  diff[j] = {d, 0, 0} for a part,
 * {dx, dy, 0} for a piece, {dx, dy, dz} for a box; each component is taken modulo
 * the lifted size of its axis.  Rows are numbered like the calculators' tables:
 * x * My + y for a piece, (x * My + y) * Mz + z for a box. */
typedef struct gg_lift_edit {
    int32_t count;
    int32_t row[4];
    int32_t slot[4];
    int32_t diff[4][3];
} gg_lift_edit;

gg_status gg_lift_create(int N, int M, int degree, int device, gg_lift **out);
gg_status gg_lift_create_piece(int Nx, int Ny, int Mx, int My, int degree, int device, gg_lift **out);
gg_status gg_lift_create_box(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, int device,
                             gg_lift **out);
/* The base table: M * degree int32 diffs (part), Mx*My * degree * 2 (piece),
 * Mx*My*Mz * degree * 3 (box); padding slots: diff 0. */
gg_status gg_lift_set_base(gg_lift *h, const int32_t *table);
/* Exact counts of each candidate over the M orbit representatives: out[i].total =
 * sum of distances from the representatives (unscaled: the reference's ASPL is
 * total * (N/M) / (N*(N-1)), cudaASPLconv.cu:241-242, with N and M the vertex and
 * representative counts), .reached = (representative, vertex) pairs reached (M*N
 * when connected), .levels = last level that found a pair.  max_levels caps the
 * BFS (0 = no cap); a candidate still finding pairs at the cap reports
 * connected = 0. */
gg_status gg_lift_eval(gg_lift *h, int n_cand, const gg_lift_edit *edits, int max_levels,
                       gg_cand_result *out);
/* Candidates that run side by side in one round (1..32; 0 = automatic: as many as
 * keep the round's bitsets within half of the L2). */
gg_status gg_lift_set_group(gg_lift *h, int group);
gg_status gg_lift_group(gg_lift *h, int *group);
/* Autotuner: times `trials` evaluations of the edits for each group size, keeps the
 * fastest as this handle's automatic group and records it in the tuning cache
 * (gg_set_tune_cache) for lifts of the same form, sizes and degree created later on
 * the same kind of GPU.  best_group / best_ms may be NULL. */
gg_status gg_lift_autotune(gg_lift *h, int n_cand, const gg_lift_edit *edits, int max_levels, int trials,
                           int *best_group, double *best_ms);
/* Tuning: past half_ppm parts per million of a round's pairs reached, a chunk
 * gathers half its neighbours first and the rest only while it still misses
 * sources (default 850000; 1000000 = never). */
gg_status gg_lift_set_half_ppm(gg_lift *h, int half_ppm);
/* Device clock (ns) at the start ([0]) and at the end of each level ([L]) of the
 * last evaluation's first round; entries past the levels run are 0. */
gg_status gg_lift_last_level_ns(gg_lift *h, uint64_t *ns, int n);
/* Device milliseconds of the last gg_lift_eval (table build and BFS launch). */
gg_status gg_lift_last_ms(gg_lift *h, double *ms);
gg_status gg_lift_destroy(gg_lift *h);

/* Random moves of a lift, the two the reference's lifted annealers draw
 * (cppcode/annealing.cpp:112-197, pieceannealing.cpp:113-204,
 * boxHillClimb.cpp:113-220): with probability 1/2 when the lift has more than one
 * copy of the orbit tile, a new lift shift for one orbit edge (2 slots); otherwise
 * an orbit 2-opt, edges a-b and c-d rewired to a-d and b-c, each with a uniform new
 * lift shift (4 slots).  Padding slots (diff 0) are never moved, and moves that
 * would give the lift a loop or a repeated edge are redrawn (the reference keeps
 * them).  The table must be symmetric (every slot has its reverse slot in the
 * target orbit's row). */
gg_status gg_gen_lift_moves(int N, int M, int degree, const int32_t *diffs, int count, uint64_t seed,
                            gg_lift_edit *out);
gg_status gg_gen_piece_moves(int Nx, int Ny, int Mx, int My, int degree, const int32_t *vals, int count,
                             uint64_t seed, gg_lift_edit *out);
gg_status gg_gen_box_moves(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, const int32_t *vals,
                           int count, uint64_t seed, gg_lift_edit *out);

/* Uniform random 2-opt proposals on a base graph (adj n*degree, simple):
 * edges (a,b), (c,d) drawn uniformly, mode uniform; proposals that would create a
 * loop or a repeated edge are redrawn.  Writes `count` swaps with base = base_id. */
gg_status gg_gen_swaps(int n, int degree, const int32_t *adj, int base_id, int count, uint64_t seed,
                       gg_swap *out);

/* ---- surrogate ΔASPL ranker (no reference counterpart) -------------------
 * A message-passing network over the current graph that predicts, for a 2-opt
 * swap, the change of the all-pairs total it would cause; trained online on
 * exact results.  It only ranks proposals: exact BFS decides everything else.
 *   x_v          per-vertex input features (in_features floats; e.g. the distance
 *                histogram of gg_batch_vertex_hist, standardised)
 *   H0 = relu(X W_in + b_in)                                    (in -> 64)
 *   H_l = relu(H_{l-1} Ws_l + mean_{u~v} H_{l-1}[u] Wn_l + b_l)  l = 1..3 (64 -> 64)
 *   swap (a,b,c,d,mode), new partners p,q ((c,d) for mode 0, (d,c) for mode 1):
 *   z = [Ha+Hb+Hc+Hd, Ha*Hb + Hc*Hd, Ha*Hp + Hb*Hq]             (192)
 *   y = relu(z Wr1 + br1) . wr2 + br2                             (prediction)
 * Weights are kept in fp32 (Adam state too) and rounded to bf16 for every
 * product; products accumulate in fp32 (mma.sync m16n8k16 bf16).  The loss is
 * the mean squared error over the swaps of a training call. */
typedef struct gg_surrogate gg_surrogate;
gg_status gg_surrogate_create(int device, int n, int degree, int in_features, uint64_t seed,
                              gg_surrogate **out);
/* Current graph (n*degree int32, symmetric) and its features (n*in_features). */
gg_status gg_surrogate_set_graph(gg_surrogate *s, const int32_t *adj, const float *features);
/* Predictions for P swaps (host arrays). */
gg_status gg_surrogate_predict(gg_surrogate *s, int P, const gg_swap *swaps, float *pred);
/* One Adam step on P (swap, target) pairs; swaps with mask[i] == 0 are ignored
 * (mask may be NULL).  *loss = the mean squared error before the step. */
gg_status gg_surrogate_train(gg_surrogate *s, int P, const gg_swap *swaps, const float *target,
                             const int32_t *mask, float lr, float *loss);
/* Parameters as one flat fp32 vector (layout: W_in, b_in, {Ws, Wn, b} x 3,
 * Wr1, br1, wr2, br2; matrices row-major [in][out]); count = number of floats. */
gg_status gg_surrogate_param_count(gg_surrogate *s, int *count);
gg_status gg_surrogate_get_params(gg_surrogate *s, float *params);
gg_status gg_surrogate_set_params(gg_surrogate *s, const float *params);
/* Gradient of the loss (same layout) without updating the parameters. */
gg_status gg_surrogate_grad(gg_surrogate *s, int P, const gg_swap *swaps, const float *target,
                            const int32_t *mask, float *grad, float *loss);
gg_status gg_surrogate_destroy(gg_surrogate *s);

/* ---- generators (host, deterministic, no GPU) ----------------------------
 * Random simple connected d-regular graph on n vertices: configuration-model
 * stub pairing followed by double-edge switches that remove loops and
 * multi-edges, retried until connected.  adj: n*d, rows sorted ascending. */
gg_status gg_gen_random_regular(int n, int d, uint64_t seed, int32_t *adj);
/* Random simple connected cyclic lift: quotient on m orbit vertices, degree d,
 * voltages in Z_g.  Output in the part form of cudaASPLconv: N = m*g, M = m,
 * diffs m*d with diff = (v-u) + m*s for the quotient edge (u,v,s) and -diff on
 * the reverse end. */
gg_status gg_gen_cyclic_lift(int m, int g, int d, uint64_t seed, int32_t *diffs);
/* Simple connected random 2-D torus lift: orbit tile Mx x My, lifted size
 * (Mx*kx) x (My*ky), degree d; vals: Mx*My * d * 2 int32 (the piece table). */
gg_status gg_gen_piece_lift(int Mx, int My, int kx, int ky, int d, uint64_t seed, int32_t *vals);

const char *gg_status_str(gg_status s);
/* Text of the last error raised on this host thread ("" if none). */
const char *gg_last_error(void);
int gg_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GG_H_ */
